// Device helpers shared by the two fused-step implementations (kernels.cu:
// triangle kernel + node kernel; cluster.cu: cluster-tiled kernel + halo
// kernel), so both apply exactly the same per-node arithmetic.
#pragma once

#include <climits>
#include <type_traits>

#include "internal.cuh"

namespace msb {
namespace stepdev {

// Buffer selection without indexing the by-value parameter arrays (a dynamic
// index would spill the whole struct to local memory).
__device__ __forceinline__ double* pos_buf(const DevState& s, int p) { return p ? s.pos[1] : s.pos[0]; }
__device__ __forceinline__ double* vel_buf(const DevState& s, int p) { return p ? s.vel[1] : s.vel[0]; }

__device__ __forceinline__ int global_step(const DevError* e, int local) {
    return *((volatile const int*)&e->base) + local;
}
// True when an earlier step of this launch tripped the force guard; such a
// step's input state must survive, so later kernels do nothing.
__device__ __forceinline__ bool stale(const DevError* e, int gstep) {
    const unsigned long long key = *((volatile const unsigned long long*)&e->guard_key);
    return key < ((unsigned long long)(unsigned)gstep << 32);
}

__device__ __forceinline__ void record_guard(const DevState& s, int gstep, long long dof) {
    const unsigned long long key = ((unsigned long long)(unsigned)gstep << 32) | (unsigned long long)dof;
    atomicMin(&s.err->guard_key, key);
    atomicExch(&s.err->flag, 3);  // MS_ERR_IMPLAUSIBLE_FORCE
}

// Larger value wins; on equal values the smaller node id wins
// (std::max_element returns the first maximum).  NaN never wins a
// comparison, as in std::max_element.
__device__ __forceinline__ void eq_merge(double& f, int& fn, double of, int ofn) {
    if (of > f || (of == f && ofn < fn)) {
        f = of;
        fn = ofn;
    }
}

// Block-wide max/argmax of |F| and |v|; the result is valid in thread 0.
// BLOCK is the block size (a multiple of 32, at most 1024).
template <int BLOCK>
__device__ __forceinline__ EqPartial eq_block_reduce(double fmax, int fnode, double vmax, int vnode) {
    __shared__ double sf[BLOCK / 32], sv[BLOCK / 32];
    __shared__ int sfn[BLOCK / 32], svn[BLOCK / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double of = __shfl_down_sync(0xffffffffu, fmax, o);
        const int ofn = __shfl_down_sync(0xffffffffu, fnode, o);
        const double ov = __shfl_down_sync(0xffffffffu, vmax, o);
        const int ovn = __shfl_down_sync(0xffffffffu, vnode, o);
        eq_merge(fmax, fnode, of, ofn);
        eq_merge(vmax, vnode, ov, ovn);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sf[warp] = fmax;
        sfn[warp] = fnode;
        sv[warp] = vmax;
        svn[warp] = vnode;
    }
    __syncthreads();
    EqPartial r{-1.0, -1.0, INT_MAX, INT_MAX};
    if (threadIdx.x == 0) {
        r = {sf[0], sv[0], sfn[0], svn[0]};
        for (int w = 1; w < BLOCK / 32; ++w) {
            eq_merge(r.f, r.fn, sf[w], sfn[w]);
            eq_merge(r.v, r.vn, sv[w], svn[w]);
        }
    }
    return r;
}

// Thread 0 of each block stores its partial at eq_part[slot] and counts; the
// last of `counted` blocks folds eq_part[0 .. total) in index order.
__device__ __forceinline__ void eq_store_and_fold(const DevState& s, const EqPartial& r, int slot, unsigned counted,
                                                  int total) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        s.eq_part[slot] = r;
        __threadfence();
        const unsigned done = atomicAdd(s.eq_counter, 1u);
        last = (done == counted - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double F = -1.0, V = -1.0;
        int Fn = INT_MAX, Vn = INT_MAX;
        for (int b = 0; b < total; ++b) {
            const volatile EqPartial* p = s.eq_part + b;
            eq_merge(F, Fn, p->f, p->fn);
            eq_merge(V, Vn, p->v, p->vn);
        }
        s.equil->max_force = F;
        s.equil->max_speed = V;
        s.equil->max_force_node = Fn;
        s.equil->max_speed_node = Vn;
        *s.eq_counter = 0u;
    }
}

// A node's state as the step reads it: position and velocity from the
// step's buffer, dof mass, constraint flag.
struct NodeIn {
    double px, py, pz, vx, vy, vz, mass;
    int fixed;
};

__device__ __forceinline__ NodeIn node_load(const DevMesh& m, const DevState& s, const StepScalars& sc, int n) {
    const int N = m.N;
    const double* pos = pos_buf(s, sc.parity);
    const double* vel = vel_buf(s, sc.parity);
    NodeIn in;
    in.px = pos[n];
    in.py = pos[N + n];
    in.pz = pos[2 * N + n];
    in.vx = vel[n];
    in.vy = vel[N + n];
    in.vz = vel[2 * N + n];
    in.mass = __ldg(m.mass + n);
    in.fixed = __ldg(m.fixed + n);
    return in;
}

// Everything after the deformation-force sum for one node: damping
// (calc_non_deformation_forces.cpp:44-57), constraints (impose_constraints.cpp:56-68),
// the equilibrium maxima (is_at_equilibrium.cpp:62-76), the force guard and
// the symplectic-Euler update (advance_dynamics.cpp:58-93) into the other
// ping-pong buffer, from the node's loaded state.
__device__ __forceinline__ void node_core(const DevMesh& m, const DevState& s, const StepScalars& sc, int gstep,
                                          int n, const NodeIn& in, double Fx, double Fy, double Fz, double& fmax,
                                          int& fnode, double& vmax, int& vnode) {
    const int N = m.N;
    const double vx = in.vx, vy = in.vy, vz = in.vz;
    const double mass = in.mass;
    if (!sc.gd) {
        // One division per node: -damping m / (rho h^2), then per component.
        const double dm = -sc.damping * mass / sc.rho_hh;
        Fx += dm * vx;
        Fy += dm * vy;
        Fz += dm * vz;
    }
    if (in.fixed) Fx = Fy = Fz = 0.0;
    if (sc.check) {
        eq_merge(fmax, fnode, sqrt(Fx * Fx + Fy * Fy + Fz * Fz), n);
        eq_merge(vmax, vnode, sqrt(vx * vx + vy * vy + vz * vz), n);
    }
    const double lim = sc.force_limit;
    if (!(fabs(Fx) < lim)) record_guard(s, gstep, (long long)n);
    if (!(fabs(Fy) < lim)) record_guard(s, gstep, (long long)N + n);
    if (!(fabs(Fz) < lim)) record_guard(s, gstep, 2LL * N + n);
    double nvx, nvy, nvz;
    if (!sc.gd) {
        const double k2 = sc.dt / mass;
        nvx = vx + k2 * Fx;
        nvy = vy + k2 * Fy;
        nvz = vz + k2 * Fz;
    } else {
        const double den = sc.damping * mass;
        nvx = sc.rho_hh * Fx / den;
        nvy = sc.rho_hh * Fy / den;
        nvz = sc.rho_hh * Fz / den;
    }
    double* npos = pos_buf(s, sc.parity ^ 1);
    double* nvel = vel_buf(s, sc.parity ^ 1);
    npos[n] = in.px + sc.dt * nvx;
    npos[N + n] = in.py + sc.dt * nvy;
    npos[2 * N + n] = in.pz + sc.dt * nvz;
    nvel[n] = nvx;
    nvel[N + n] = nvy;
    nvel[2 * N + n] = nvz;
}

__device__ __forceinline__ void node_finish(const DevMesh& m, const DevState& s, const StepScalars& sc, int gstep,
                                            int n, double Fx, double Fy, double Fz, double& fmax, int& fnode,
                                            double& vmax, int& vnode) {
    node_core(m, s, sc, gstep, n, node_load(m, s, sc, n), Fx, Fy, Fz, fmax, fnode, vmax, vnode);
}

// Entries whose indices, then contributions, one thread loads together.
#ifndef MSB_NODE_PREFETCH
#define MSB_NODE_PREFETCH 1
#endif
#ifndef MSB_NODE_BATCH
#define MSB_NODE_BATCH 3
#endif
constexpr int kNodeBatch = MSB_NODE_BATCH;

// Sum of node n's contributions in entry order over the sliced lists: the
// warp's slice header is one broadcast load, entry indices load coalesced
// (entry k of the 32 nodes is 128 contiguous bytes), and kNodeBatch
// indices, then their contributions, are in flight at once.  The loop
// bound (the slice width) is uniform over the warp.
template <typename Cf>
__device__ __forceinline__ void gather_sell(const DevMesh& m, const Cf* __restrict__ c, int n, double& Fx,
                                            double& Fy, double& Fz) {
    const int w = n >> 5, lane = n & 31;
    const int base = __ldg(m.sell_off + w);
    const int width = (__ldg(m.sell_off + w + 1) - base) >> 5;
    const int* __restrict__ ep = m.sell_ent + base + lane;
#if MSB_NODE_PREFETCH
    // The next batch's entry ids load together with this batch's
    // contributions, so each batch costs one round trip, not two.
    int nx[kNodeBatch];
#pragma unroll
    for (int j = 0; j < kNodeBatch; ++j) nx[j] = (j < width) ? __ldg(ep + 32 * j) : -1;
#endif
    for (int k = 0; k < width; k += kNodeBatch) {
        int ei[kNodeBatch];
#if MSB_NODE_PREFETCH
#pragma unroll
        for (int j = 0; j < kNodeBatch; ++j) {
            ei[j] = nx[j];
            const int kk = k + kNodeBatch + j;
            nx[j] = (kk < width) ? __ldg(ep + 32 * kk) : -1;
        }
#else
#pragma unroll
        for (int j = 0; j < kNodeBatch; ++j) ei[j] = (k + j < width) ? __ldg(ep + 32 * (k + j)) : -1;
#endif
        Cf v[kNodeBatch][3];
        constexpr int S = std::is_same<Cf, float>::value ? kMixedSlot : 3;
#pragma unroll
        for (int j = 0; j < kNodeBatch; ++j) {
            if (ei[j] >= 0) {
                const Cf* q = c + S * (size_t)ei[j];
                if constexpr (S == 4) {
                    const float4 w = __ldg(reinterpret_cast<const float4*>(q));
                    v[j][0] = w.x;
                    v[j][1] = w.y;
                    v[j][2] = w.z;
                } else {
                    v[j][0] = q[0];
                    v[j][1] = q[1];
                    v[j][2] = q[2];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kNodeBatch; ++j) {
            if (ei[j] >= 0) {
                Fx += (double)v[j][0];
                Fy += (double)v[j][1];
                Fz += (double)v[j][2];
            }
        }
    }
}

}  // namespace stepdev
}  // namespace msb
