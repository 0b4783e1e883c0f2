// Batched ensembles (ms_batch_* in include/morphoshell_gpu.h).
//
// The instances' tables are concatenated into one union mesh; every step is
// k_batch_pre, the force step (k_batch_node_tiles alone, the node-tiled
// schedule, or k_batch_tri / k_batch_tri_tiles then k_batch_node) and
// k_batch_post over the whole union:
//   k_batch_pre   one thread per instance: the top of main.cpp's loop body
//                 (dial factor clamp :286-288, end of a dial phase :293-304,
//                 whether this step checks for equilibrium) and the
//                 protocol-3 values of this step (do_dialling.cpp:112-123)
//   k_batch_tri   one thread per triangle: the per-triangle contributions of
//                 the two-kernel step with the instance's material and dial
//                 values
//   k_batch_node  one thread per node: the deterministic gather, damping,
//                 constraints, per-node |F| and |v| on check steps, the force
//                 guard and the symplectic-Euler update, with the instance's
//                 timestep and damping
//   k_batch_post  one block per instance: the equilibrium test over the
//                 instance's nodes (is_at_equilibrium.cpp:62-98), a guard
//                 trip, and the end of the loop body (main.cpp:476-507)
// Done and failed instances are skipped by every kernel and keep their state
// in the ping-pong buffer recorded in InstState::frozen_parity.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/morphoshell_gpu.h"
#include "internal.cuh"
#include "node_tile_walk.cuh"
#include "step_common.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace {

using namespace stepdev;
using namespace tridev;

__device__ __forceinline__ bool is_frozen(int status) { return status >= INST_DONE; }

// Material of triangle t of an instance: the instance's uniform material
// (coefficients formed on the host) or the triangle's own.
__device__ __forceinline__ void inst_material(const InstParams& q, const DevMesh& m, int t, TriMat<double>& mt) {
    if (q.uniform_hmu) {
        mt.h = q.h;
        mt.mu = q.mu;
        mt.ks = q.ks;
        mt.kb = q.kb;
        mt.igmh = q.igmh;
    } else {
        set_material(__ldg(m.thick + t), __ldg(m.shear + t), q.nu, q.gamma, mt);
    }
}

__global__ void k_batch_pre(const InstParams* __restrict__ ip, InstState* __restrict__ is, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    InstState st = is[i];
    if (is_frozen(st.status)) return;
    const InstParams& p = ip[i];
    if (st.dial_factor >= 1.0) st.dial_factor = 1.0;
    if (st.status == INST_DIALLING && st.k_phase >= p.steps_per_phase) {
        st.status = INST_WAITING;
        st.tsc = 0;
        st.damping = p.damping2;
    }
    st.check_now = (st.status == INST_WAITING && st.tsc > p.steps_between_checks) ? 1 : 0;
    if (st.status == INST_DIALLING) {
        const double d = st.dial_factor;
        const double lam = (1.0 - d) * 1.0 + d * p.lam_final;
        st.cur_dial = d;
        st.cur_lam = lam;
        st.cur_pw = pow(lam, -2.0 * p.nu_ot);
    }
    is[i] = st;
}

template <bool MIXED, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_tri(const DevMesh m, const ClusterPlan p, const DevState s,
                                                     const InstParams* __restrict__ ip,
                                                     const InstState* __restrict__ is, int parity) {
    using R = typename Real<MIXED>::T;
    constexpr int CS = contrib_stride<MIXED>();
    __shared__ R stage[BLOCK * CS];
    const int t = blockIdx.x * BLOCK + threadIdx.x;
    const bool live = t < m.T;
    R f[18];
#pragma unroll
    for (int j = 0; j < 18; ++j) f[j] = R(0);
    if (live) {
        const int4 a = __ldg(p.tri_idx + 2 * t);
        const int4 b = __ldg(p.tri_idx + 2 * t + 1);
        const int inst = b.w;
        const InstState& st = is[inst];
        if (!is_frozen(st.status)) {
            const InstParams& q = ip[inst];
            TriMat<double> mt;
            inst_material(q, m, t, mt);
            const int ids[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
            tri_contrib<DIAL_LCE, MIXED>(m, p, pos_buf(s, parity), t, ids, st.cur_dial, st.cur_lam, st.cur_pw, f,
                                         q.nu, mt);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (!__any_sync(0xffffffffu, live)) return;
    R* sw = stage + warp * 32 * CS;
    stage_contrib<MIXED>(sw + lane * CS, f);
    __syncwarp();
    const int t0 = t - lane;
    const int total = min(32, m.T - t0) * CS;
    R* out;
    if constexpr (MIXED) out = m.contrib_f + (size_t)t0 * CS;
    else out = s.contrib + (size_t)t0 * CS;
    for (int j = lane; j < total; j += 32) out[j] = sw[j];
}

// One triangle of a tile or chunk record with its instance's material and
// protocol-3 values (nothing for a done or failed instance).  Shared by the
// tile and node-tile kernels, so they give the same bits.
template <bool MIXED>
__device__ __forceinline__ void batch_tri(const DevMesh& m, const int* __restrict__ tri_inst,
                                          const InstParams* __restrict__ ip, const InstState* __restrict__ is,
                                          const double* __restrict__ pos, int t, int inst_hint, const int (&ids)[6],
                                          const typename Real<MIXED>::T (&c)[24], double area, double c2, double s2,
                                          double cs, typename Real<MIXED>::T (&f)[18]) {
    // The gathers go first: they do not depend on the instance, so they are
    // in flight while its id and state load (a frozen instance's positions
    // are read and not used).
    double P[6][3];
#pragma unroll
    for (int sl = 0; sl < 6; ++sl) {
        P[sl][0] = __ldg(pos + ids[sl]);
        P[sl][1] = __ldg(pos + m.N + ids[sl]);
        P[sl][2] = __ldg(pos + 2 * m.N + ids[sl]);
    }
    const int inst = inst_hint >= 0 ? inst_hint : __ldg(tri_inst + t);
    const InstState& st = is[inst];
    if (is_frozen(st.status)) return;
    const InstParams& q = ip[inst];
    TriMat<double> mt;
    inst_material(q, m, t, mt);
    mt.area = area;
    lce_metric(c2, s2, cs, __dmul_rn(st.cur_lam, st.cur_lam), st.cur_pw, mt);
    tri_forces<MIXED>(P, c, mt, q.nu, f);
}

// The same contributions from bulk-copied tile records (tile_copy.cuh),
// persistent blocks; tri_inst[t] is the triangle's instance.
template <bool MIXED>
__global__ void __launch_bounds__(kTile) k_batch_tri_tiles(const DevMesh m, const ClusterPlan p, const DevState s,
                                                         const int* __restrict__ tri_inst,
                                                         const InstParams* __restrict__ ip,
                                                         const InstState* __restrict__ is, int* err, int parity) {
    using R = typename Real<MIXED>::T;
    const double* pos = pos_buf(s, parity);
    const unsigned char* tl = reinterpret_cast<const unsigned char*>(MIXED ? p.tiles_f : p.tiles);
    R* out;
    if constexpr (MIXED) out = m.contrib_f;
    else out = s.contrib;
    tiles::tile_loop<MIXED>(
        m.T, tl, out, err,
        [&](int t, const int (&ids)[6], const R (&c)[24], double area, double c2, double s2, double cs, R (&f)[18]) {
            batch_tri<MIXED>(m, tri_inst, ip, is, pos, t, -1, ids, c, area, c2, s2, cs, f);
        });
}

// Everything after the deformation-force sum for node n of a live instance:
// node_finish with the instance's scalars, |F| and |v| to fnorm / vnorm on
// the instance's check steps, a guard trip into the instance's guard key.
// A node's state for the update: position and velocity from buffer
// `parity`, mass, constraint flag (independent of its instance, so these
// loads can be in flight while the instance's state loads).
__device__ __forceinline__ NodeIn batch_node_load(const DevMesh& m, const DevState& s, int n, int parity) {
    const int N = m.N;
    const double* pos = pos_buf(s, parity);
    const double* vel = vel_buf(s, parity);
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

__device__ __forceinline__ void batch_node_core(const DevMesh& m, const DevState& s, const InstParams& q,
                                                InstState* __restrict__ is, int inst, int n, const NodeIn& in,
                                                double Fx, double Fy, double Fz, double* __restrict__ fnorm,
                                                double* __restrict__ vnorm, int parity) {
    const int N = m.N;
    const double damping = is[inst].damping;
    const int check = is[inst].check_now;
    const double vx = in.vx, vy = in.vy, vz = in.vz;
    const double mass = in.mass;
    const double dm = -damping * mass / q.rho_hh;
    Fx += dm * vx;
    Fy += dm * vy;
    Fz += dm * vz;
    if (in.fixed) Fx = Fy = Fz = 0.0;
    if (check) {
        fnorm[n] = sqrt(Fx * Fx + Fy * Fy + Fz * Fz);
        vnorm[n] = sqrt(vx * vx + vy * vy + vz * vz);
    }
    const double lim = q.force_limit;
    const long long Ni = q.node_end - q.node_begin, ln = n - q.node_begin;
    if (!(fabs(Fx) < lim)) atomicMin(&is[inst].guard_key, (unsigned long long)ln);
    if (!(fabs(Fy) < lim)) atomicMin(&is[inst].guard_key, (unsigned long long)(Ni + ln));
    if (!(fabs(Fz) < lim)) atomicMin(&is[inst].guard_key, (unsigned long long)(2 * Ni + ln));
    const double k2 = q.dt / mass;
    const double nvx = vx + k2 * Fx, nvy = vy + k2 * Fy, nvz = vz + k2 * Fz;
    double* npos = pos_buf(s, parity ^ 1);
    double* nvel = vel_buf(s, parity ^ 1);
    npos[n] = in.px + q.dt * nvx;
    npos[N + n] = in.py + q.dt * nvy;
    npos[2 * N + n] = in.pz + q.dt * nvz;
    nvel[n] = nvx;
    nvel[N + n] = nvy;
    nvel[2 * N + n] = nvz;
}

template <bool MIXED, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_node(const DevMesh m, const DevState s,
                                                      const int* __restrict__ node_inst,
                                                      const InstParams* __restrict__ ip, InstState* __restrict__ is,
                                                      double* __restrict__ fnorm, double* __restrict__ vnorm,
                                                      int parity) {
    const int n = blockIdx.x * BLOCK + threadIdx.x;
    const int N = m.N;
    int inst = 0;
    bool active = false;
    if (n < N) {
        inst = __ldg(node_inst + n);
        active = !is_frozen(is[inst].status);
    }
    if (!__any_sync(0xffffffffu, active)) return;  // warp-uniform
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    if constexpr (MIXED) gather_sell<float>(m, m.contrib_f, n, Fx, Fy, Fz);
    else gather_sell<double>(m, s.contrib, n, Fx, Fy, Fz);
    if (!active) return;
    batch_node_core(m, s, ip[inst], is, inst, n, batch_node_load(m, s, n, parity), Fx, Fy, Fz, fnorm, vnorm, parity);
}

// The whole step of the union in one kernel (node_tile_walk.cuh): a block
// sums the forces of its tiles of nodes in shared memory, computing every
// triangle that touches them, and updates the tiles' live nodes.
#ifndef MSB_NT_MINB
#define MSB_NT_MINB 3
#endif
#ifndef MSB_NT_MINB_MIXED
#define MSB_NT_MINB_MIXED 4
#endif
template <bool MIXED>
__global__ void __launch_bounds__(kTile, MIXED ? MSB_NT_MINB_MIXED : MSB_NT_MINB)
    k_batch_node_tiles(const DevMesh m, const NodeTilePlan q, const DevState s, const int* __restrict__ tri_inst,
                       const int* __restrict__ node_inst, const InstParams* __restrict__ ip,
                       InstState* __restrict__ is, double* __restrict__ fnorm, double* __restrict__ vnorm, int* err,
                       int parity) {
    using R = typename Real<MIXED>::T;
    const double* pos = pos_buf(s, parity);
    tiles::node_tile_walk<MIXED>(
        q, m.N, true, err,
        [&](int t, int inst, const int (&ids)[6], const R (&c)[24], double area, double c2, double s2, double cs,
            R (&f)[18]) { batch_tri<MIXED>(m, tri_inst, ip, is, pos, t, inst, ids, c, area, c2, s2, cs, f); },
        [&](int n, double Fx, double Fy, double Fz) {
            const NodeIn in = batch_node_load(m, s, n, parity);  // read for frozen instances too, then unused
            const int inst = __ldg(node_inst + n);
            if (!is_frozen(is[inst].status))
                batch_node_core(m, s, ip[inst], is, inst, n, in, Fx, Fy, Fz, fnorm, vnorm, parity);
        });
}

// The tables part of the node-tiled records (ids, weights, area and
// director trigonometry, field-major per chunk), gathered from the union's
// per-triangle tables: the bytes fill_node_tile_records writes on the host;
// and each slot's instance (the plan's chunk_tag, which the walk loads with
// the tables).  One block per chunk, one thread per slot; empty slots get
// zeros.
template <bool MIXED>
__global__ void __launch_bounds__(kTile)
    k_fill_node_tile_tables(unsigned char* __restrict__ rec, size_t stride, const int* __restrict__ chunk_tri,
                            const int4* __restrict__ tri_idx, const typename Real<MIXED>::T* __restrict__ coef,
                            const double4* __restrict__ aux, int* __restrict__ chunk_inst) {
    using R = typename Real<MIXED>::T;
    using L = tiles::TileLayout<MIXED>;
    const int c = blockIdx.x, i = threadIdx.x;
    unsigned char* r = rec + (size_t)c * stride;
    int* ids = reinterpret_cast<int*>(r);
    R* cf = reinterpret_cast<R*>(r + L::ids);
    double* ax = reinterpret_cast<double*>(r + L::ids + L::coef);
    const int t = chunk_tri[(size_t)c * kTile + i];
    if (t >= 0) {
        const int4 a = tri_idx[2 * (size_t)t], b = tri_idx[2 * (size_t)t + 1];
        chunk_inst[(size_t)c * kTile + i] = b.w;  // the triangle's instance
        const int id[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
#pragma unroll
        for (int k = 0; k < 6; ++k) ids[k * kTile + i] = id[k];
#pragma unroll
        for (int k = 0; k < 24; ++k) cf[k * kTile + i] = coef[24 * (size_t)t + k];
        const double4 x = aux[t];
        ax[i] = x.x;
        ax[kTile + i] = x.y;
        ax[2 * kTile + i] = x.z;
        ax[3 * kTile + i] = x.w;
    } else {
        chunk_inst[(size_t)c * kTile + i] = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k) ids[k * kTile + i] = 0;
#pragma unroll
        for (int k = 0; k < 24; ++k) cf[k * kTile + i] = R(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) ax[k * kTile + i] = 0.0;
    }
}

constexpr int kPostBlock = 256;

__global__ void __launch_bounds__(kPostBlock) k_batch_post(const InstParams* __restrict__ ip,
                                                           InstState* __restrict__ is,
                                                           const double* __restrict__ fnorm,
                                                           const double* __restrict__ vnorm, int parity) {
    const int i = blockIdx.x;
    const InstParams& p = ip[i];
    const int status = is[i].status;
    if (is_frozen(status)) return;  // uniform over the block
    const bool guard = is[i].guard_key != ~0ULL;
    const bool check = is[i].check_now != 0;
    EqPartial r{-1.0, -1.0, INT_MAX, INT_MAX};
    if (check && !guard) {  // uniform
        double fm = -1.0, vm = -1.0;
        int fn = INT_MAX, vn = INT_MAX;
        for (int n = p.node_begin + threadIdx.x; n < p.node_end; n += kPostBlock) {
            eq_merge(fm, fn, fnorm[n], n - p.node_begin);
            eq_merge(vm, vn, vnorm[n], n - p.node_begin);
        }
        r = eq_block_reduce<kPostBlock>(fm, fn, vm, vn);
    }
    if (threadIdx.x != 0) return;
    InstState st = is[i];
    if (guard) {
        // The state before this step survives in the buffer it read
        // (main.cpp:448-474 stops the run there).
        st.status = INST_FAILED;
        st.frozen_parity = parity;
        is[i] = st;
        return;
    }
    if (check) {
        st.max_force = r.f;
        st.max_speed = r.v;
        st.max_force_node = r.fn;
        st.max_speed_node = r.vn;
        if ((r.f / p.char_force) < p.force_thresh && (r.v / p.char_speed) < p.speed_thresh) {
            st.status = INST_EQUIL;
            st.equilibria += 1;
            st.last_equil_dial = st.dial_factor;
        }
        st.tsc = 0;
    }
    st.time += p.dt;
    st.stepcount += 1;
    if (st.status == INST_DIALLING) st.k_phase += 1;
    st.dial_factor = st.last_equil_dial + p.spacing * ((double)st.k_phase / (double)p.steps_per_phase);
    if (st.status == INST_WAITING) st.tsc += 1;
    if (st.status == INST_EQUIL && st.last_equil_dial >= 1.0 && p.stop_at_final) {
        st.status = INST_DONE;
        st.frozen_parity = parity ^ 1;
        st.dial_factor = st.last_equil_dial;
    } else if (st.status == INST_EQUIL) {
        st.status = INST_DIALLING;
        st.k_phase = 0;
        st.damping = p.damping1;
    }
    is[i] = st;
}

// ---- schedules ------------------------------------------------------------------

struct Sched {
    int tri_block, node_block;
};
// tri_block -1: the node-tiled one-kernel step (node_block unused); 0: the
// persistent bulk-copy tile kernel.
constexpr int kSchedNodeTiles = 0, kSchedTiles = 1, kSchedAos = 2;
constexpr Sched kScheds[] = {{-1, 0},    {0, 256},   {128, 256}, {64, 256}, {256, 256},
                             {128, 128}, {64, 128},  {256, 128}, {128, 512}, {0, 128}};
constexpr int kNumScheds = sizeof(kScheds) / sizeof(kScheds[0]);

template <bool MIXED>
cudaError_t launch_tri(int tb, const DevMesh& m, const ClusterPlan& p, const DevState& s, const InstParams* ip,
                       const InstState* is, int parity, cudaStream_t st) {
    const int T = m.T;
    switch (tb) {
        case 64: k_batch_tri<MIXED, 64><<<(T + 63) / 64, 64, 0, st>>>(m, p, s, ip, is, parity); break;
        case 128: k_batch_tri<MIXED, 128><<<(T + 127) / 128, 128, 0, st>>>(m, p, s, ip, is, parity); break;
        case 256: k_batch_tri<MIXED, 256><<<(T + 255) / 256, 256, 0, st>>>(m, p, s, ip, is, parity); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <bool MIXED>
cudaError_t launch_node(int nb, const DevMesh& m, const DevState& s, const int* node_inst, const InstParams* ip,
                        InstState* is, double* fnorm, double* vnorm, int parity, cudaStream_t st) {
    const int N = m.N;
    switch (nb) {
        case 128:
            k_batch_node<MIXED, 128><<<(N + 127) / 128, 128, 0, st>>>(m, s, node_inst, ip, is, fnorm, vnorm, parity);
            break;
        case 256:
            k_batch_node<MIXED, 256><<<(N + 255) / 256, 256, 0, st>>>(m, s, node_inst, ip, is, fnorm, vnorm, parity);
            break;
        case 512:
            k_batch_node<MIXED, 512><<<(N + 511) / 512, 512, 0, st>>>(m, s, node_inst, ip, is, fnorm, vnorm, parity);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace
}  // namespace msb

using namespace msb;

namespace {

struct BatchGraph {
    int len, parity, sched;
    cudaGraphExec_t exec;
};

}  // namespace

struct ms_batch {
    int device = 0;
    int precision = 0;
    cudaStream_t stream = nullptr;
    DevMesh m{};
    ClusterPlan p{};
    DevState s{};
    int n_inst = 0;
    std::vector<InstParams> ip;
    std::vector<InstState> init_state;
    InstParams* d_ip = nullptr;
    InstState* d_is = nullptr;
    int* d_node_inst = nullptr;
    double* d_fnorm = nullptr;
    double* d_vnorm = nullptr;
    InstState* h_is = nullptr;  // pinned mirror
    int* d_tri_inst = nullptr;   // [T]
    int* d_err = nullptr;        // copy-wait timeouts of the tile kernels
    int tile_grid = 0;           // 0: tile kernel unavailable
    NodeTilePlan ntp{};          // node-tiled step over the union
    bool have_nt = false;
    int nt_blocks = 0;           // resident blocks per SM the node-tiled plan runs at
    std::string tune_report;     // the last autotune's trials, one per line
    std::vector<void*> nt_allocs;  // the node-tiled plan's device buffers (replaced by the autotuner)
    int parity = 0;
    int sched = 0;
    int chunk = 64;
    std::vector<BatchGraph> graphs;
    std::vector<void*> allocs;
    std::string last_error;
};

namespace {

ms_status bfail(ms_batch* b, ms_status st, const std::string& msg) {
    if (b) b->last_error = msg;
    return st;
}

ms_status bcuda(ms_batch* b, cudaError_t e, const char* what) {
    const std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return bfail(b, MS_ERR_OUT_OF_MEMORY, msg);
    return bfail(b, MS_ERR_CUDA, msg);
}

#define MB_CUDA(b, call)                                   \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return bcuda(b, e_, #call); \
    } while (0)

#define MB_TRY(expr)                  \
    do {                              \
        ms_status st_ = (expr);       \
        if (st_ != MS_OK) return st_; \
    } while (0)

template <typename T>
ms_status balloc(ms_batch* b, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return bcuda(b, e, "cudaMalloc");
    b->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return MS_OK;
}

template <typename T>
ms_status bupload(ms_batch* b, T** dst, const std::vector<T>& src) {
    MB_TRY(balloc(b, dst, src.size()));
    if (!src.empty()) MB_CUDA(b, cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MS_OK;
}

void clear_graphs(ms_batch* b) {
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
}

ms_status launch_step(ms_batch* b, int parity, int sched) {
    const Sched& sc = kScheds[sched];
    cudaStream_t st = b->stream;
    const int n = b->n_inst;
    k_batch_pre<<<(n + 127) / 128, 128, 0, st>>>(b->d_ip, b->d_is, n);
    cudaError_t e;
    if (sc.tri_block < 0) {
        const NodeTilePlan& q = b->ntp;
        const int grid = std::min(q.ntiles, q.grid);
        if (b->precision == MS_PRECISION_MIXED)
            k_batch_node_tiles<true><<<grid, kTile, tiles::NtSmem<true>::bytes(q.stride, q.nodes), st>>>(
                b->m, q, b->s, b->d_tri_inst, b->d_node_inst, b->d_ip, b->d_is, b->d_fnorm, b->d_vnorm, b->d_err,
                parity);
        else
            k_batch_node_tiles<false><<<grid, kTile, tiles::NtSmem<false>::bytes(q.stride, q.nodes), st>>>(
                b->m, q, b->s, b->d_tri_inst, b->d_node_inst, b->d_ip, b->d_is, b->d_fnorm, b->d_vnorm, b->d_err,
                parity);
        e = cudaGetLastError();
    } else if (sc.tri_block == 0) {
        const int ntiles = (b->m.T + kTile - 1) / kTile;
        const int grid = std::min(ntiles, b->tile_grid);
        if (b->precision == MS_PRECISION_MIXED)
            k_batch_tri_tiles<true><<<grid, kTile, 2 * tiles::TileLayout<true>::bytes, st>>>(
                b->m, b->p, b->s, b->d_tri_inst, b->d_ip, b->d_is, b->d_err, parity);
        else
            k_batch_tri_tiles<false><<<grid, kTile, 2 * tiles::TileLayout<false>::bytes, st>>>(
                b->m, b->p, b->s, b->d_tri_inst, b->d_ip, b->d_is, b->d_err, parity);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = b->precision == MS_PRECISION_MIXED
                    ? launch_node<true>(sc.node_block, b->m, b->s, b->d_node_inst, b->d_ip, b->d_is, b->d_fnorm,
                                        b->d_vnorm, parity, st)
                    : launch_node<false>(sc.node_block, b->m, b->s, b->d_node_inst, b->d_ip, b->d_is, b->d_fnorm,
                                         b->d_vnorm, parity, st);
    } else if (b->precision == MS_PRECISION_MIXED) {
        e = launch_tri<true>(sc.tri_block, b->m, b->p, b->s, b->d_ip, b->d_is, parity, st);
        if (e == cudaSuccess)
            e = launch_node<true>(sc.node_block, b->m, b->s, b->d_node_inst, b->d_ip, b->d_is, b->d_fnorm,
                                  b->d_vnorm, parity, st);
    } else {
        e = launch_tri<false>(sc.tri_block, b->m, b->p, b->s, b->d_ip, b->d_is, parity, st);
        if (e == cudaSuccess)
            e = launch_node<false>(sc.node_block, b->m, b->s, b->d_node_inst, b->d_ip, b->d_is, b->d_fnorm,
                                   b->d_vnorm, parity, st);
    }
    if (e != cudaSuccess) return bcuda(b, e, "batch step launch");
    k_batch_post<<<n, kPostBlock, 0, st>>>(b->d_ip, b->d_is, b->d_fnorm, b->d_vnorm, parity);
    MB_CUDA(b, cudaGetLastError());
    return MS_OK;
}

// Launches `len` steps starting on buffer `parity` as one graph.
ms_status run_graph(ms_batch* b, int len, int parity, int sched) {
    for (auto& g : b->graphs)
        if (g.len == len && g.parity == parity && g.sched == sched) {
            MB_CUDA(b, cudaGraphLaunch(g.exec, b->stream));
            return MS_OK;
        }
    cudaGraph_t graph;
    MB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    ms_status st = MS_OK;
    for (int k = 0; k < len && st == MS_OK; ++k) st = launch_step(b, parity ^ (k & 1), sched);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (st != MS_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return st;
    }
    MB_CUDA(b, e);
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    MB_CUDA(b, e);
    if (b->graphs.size() >= 16) clear_graphs(b);
    b->graphs.push_back({len, parity, sched, exec});
    MB_CUDA(b, cudaGraphLaunch(exec, b->stream));
    return MS_OK;
}

// Device buffers of a node-tiled plan for a layout L of NT-node tiles run
// at `blocks` resident blocks per SM: the node sections and slot triangles
// from the host, the tables gathered on the device from the union's
// per-triangle tables.  On success q describes the plan and allocs holds
// its buffers (the caller frees them).
ms_status plan_from_layout(ms_batch* b, const NodeTileLayout& L, int NT, int blocks, NodeTilePlan& q,
                           std::vector<void*>& allocs) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t pitch = L.stride - L.fixed;
    std::vector<unsigned char> sections;
    std::vector<int> ctri;
    fill_node_sections(L, pitch, sections, ctri);
    auto dal = [&](void** ptr, size_t bytes) -> ms_status {
        cudaError_t e = cudaMalloc(ptr, std::max<size_t>(bytes, 1));
        if (e != cudaSuccess) return bcuda(b, e, "cudaMalloc (node-tiled plan)");
        allocs.push_back(*ptr);
        return MS_OK;
    };
    unsigned char* d_rec;
    int *d_tc, *d_ctri, *d_tag;
    unsigned* d_bytes;
    MB_TRY(dal(reinterpret_cast<void**>(&d_rec), L.stride * (size_t)L.C));
    MB_TRY(dal(reinterpret_cast<void**>(&d_tag), sizeof(int) * ctri.size()));
    MB_TRY(dal(reinterpret_cast<void**>(&d_tc), sizeof(int) * L.tile_chunk.size()));
    MB_TRY(dal(reinterpret_cast<void**>(&d_bytes), sizeof(unsigned) * L.bytes.size()));
    MB_TRY(dal(reinterpret_cast<void**>(&d_ctri), sizeof(int) * ctri.size()));
    MB_CUDA(b, cudaMemcpy(d_tc, L.tile_chunk.data(), sizeof(int) * L.tile_chunk.size(), cudaMemcpyHostToDevice));
    MB_CUDA(b, cudaMemcpy(d_bytes, L.bytes.data(), sizeof(unsigned) * L.bytes.size(), cudaMemcpyHostToDevice));
    MB_CUDA(b, cudaMemcpy(d_ctri, ctri.data(), sizeof(int) * ctri.size(), cudaMemcpyHostToDevice));
    MB_CUDA(b, cudaMemcpy2D(d_rec + L.fixed, L.stride, sections.data(), pitch, pitch, (size_t)L.C,
                            cudaMemcpyHostToDevice));
    if (L.C > 0) {
        if (b->precision == MS_PRECISION_MIXED)
            k_fill_node_tile_tables<true><<<L.C, kTile, 0, b->stream>>>(d_rec, L.stride, d_ctri, b->p.tri_idx,
                                                                        b->p.coef_aos_f, b->p.tri_aux, d_tag);
        else
            k_fill_node_tile_tables<false><<<L.C, kTile, 0, b->stream>>>(d_rec, L.stride, d_ctri, b->p.tri_idx,
                                                                         b->p.coef_aos, b->p.tri_aux, d_tag);
        MB_CUDA(b, cudaGetLastError());
        MB_CUDA(b, cudaStreamSynchronize(b->stream));
    }
    q = NodeTilePlan{};
    q.nodes = NT;
    q.ntiles = L.K;
    q.nchunks = L.C;
    q.grid = sms * blocks;
    q.stride = L.stride;
    q.slc = L.slc_max;
    q.rec = d_rec;
    q.tile_chunk = d_tc;
    q.chunk_bytes = d_bytes;
    q.chunk_tri = d_ctri;
    q.chunk_tag = d_tag;
    return MS_OK;
}

// Resident blocks per SM of the batched node-tiled kernel at `smem` bytes of
// shared memory per block (0: it cannot run).
int batch_node_tile_blocks(int mixed, size_t smem) {
    int nb = 0;
    cudaError_t ea = mixed ? cudaFuncSetAttribute(k_batch_node_tiles<true>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                           : cudaFuncSetAttribute(k_batch_node_tiles<false>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ea == cudaSuccess)
        ea = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch_node_tiles<true>, kTile, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batch_node_tiles<false>, kTile, smem);
    if (ea != cudaSuccess) {
        cudaGetLastError();
        nb = 0;
    }
    return nb;
}

bool all_frozen(const ms_batch* b) {
    for (int i = 0; i < b->n_inst; ++i)
        if (b->h_is[i].status < INST_DONE) return false;
    return true;
}

ms_status fetch_states(ms_batch* b) {
    MB_CUDA(b, cudaMemcpyAsync(b->h_is, b->d_is, sizeof(InstState) * b->n_inst, cudaMemcpyDeviceToHost, b->stream));
    int e = 0;
    if (b->d_err) MB_CUDA(b, cudaMemcpyAsync(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    MB_CUDA(b, cudaStreamSynchronize(b->stream));
    if (e) return bfail(b, MS_ERR_TIMEOUT, "a tile copy did not land within its bounded wait");
    return MS_OK;
}

InstState initial_state(const ms_batch_instance& in) {
    InstState st{};
    st.status = INST_DIALLING;
    st.check_now = 0;
    st.equilibria = 0;
    st.frozen_parity = -1;
    // main.cpp:250-262 (timesteps_since_previous_equil_check starts at a
    // large negative value; the phase counter resumes inside the phase that
    // dial_factor_to_start_from falls in).
    st.k_phase = static_cast<long long>(std::fmod(in.dial_factor_to_start_from, in.dial_factors_to_hold_at_spacing) *
                                        static_cast<double>(in.timesteps_per_dial_phase));
    st.tsc = -123456;
    st.stepcount = 0;
    st.dial_factor = in.dial_factor_to_start_from;
    st.last_equil_dial = in.dial_factor_to_start_from;
    st.time = 0.0;
    st.damping = in.damping_factor_1;
    st.cur_dial = st.cur_lam = st.cur_pw = 0.0;
    st.max_force = st.max_speed = -1.0;
    st.max_force_node = st.max_speed_node = -1;
    st.guard_key = ~0ULL;
    return st;
}

ms_status validate(const ms_batch_instance& in, std::string& why) {
    const ms_mesh_desc& d = in.mesh;
    if (d.num_nodes <= 0 || d.num_tris <= 0 || !d.patch_ids || !d.deriv_coeffs || !d.ref_area || !d.ref_thickness ||
        !d.ref_shear_modulus || !d.node_mass || !d.is_constrained || !in.abar_info || !in.dofs) {
        why = "missing mesh table, abar_info or dofs";
        return MS_ERR_INVALID_ARGUMENT;
    }
    for (long long k = 0; k < 6LL * d.num_tris; ++k)
        if (d.patch_ids[k] < 0 || d.patch_ids[k] >= d.num_nodes) {
            why = "patch id out of range";
            return MS_ERR_INVALID_ARGUMENT;
        }
    if (!(in.timestep > 0.0) || in.timesteps_per_dial_phase <= 0 || !(in.dial_factors_to_hold_at_spacing > 0.0)) {
        why = "timestep, timesteps_per_dial_phase and dial spacing must be positive";
        return MS_ERR_INVALID_ARGUMENT;
    }
    const double lf = in.abar_info[1], nu = in.abar_info[2];
    for (int t = 0; t < d.num_tris; ++t)
        if (in.abar_info[3LL * t + 1] != lf || in.abar_info[3LL * t + 2] != nu) {
            why = "lambda_final and nu_ot must be uniform within an instance";
            return MS_ERR_UNSUPPORTED;
        }
    return MS_OK;
}

}  // namespace

extern "C" {

ms_status ms_batch_create(const ms_batch_instance* inst, int32_t n, int32_t device, int32_t precision,
                          ms_batch** out) {
    if (!out) return MS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!inst || n <= 0) return MS_ERR_INVALID_ARGUMENT;
    if (precision != MS_PRECISION_FP64 && precision != MS_PRECISION_MIXED) return MS_ERR_INVALID_ARGUMENT;
    long long N = 0, T = 0;
    for (int i = 0; i < n; ++i) {
        std::string why;
        const ms_status v = validate(inst[i], why);
        if (v != MS_OK) return v;
        N += inst[i].mesh.num_nodes;
        T += inst[i].mesh.num_tris;
    }
    if (6 * T >= (1LL << 31) || N >= (1LL << 31)) return MS_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MS_ERR_NO_DEVICE;
    if (device >= ndev) return MS_ERR_INVALID_ARGUMENT;
    if (device >= 0) cudaSetDevice(device);

    ms_batch* b = new ms_batch();
    cudaGetDevice(&b->device);
    b->precision = precision;
    b->n_inst = n;
    auto bail = [&](ms_status st) {
        ms_batch_destroy(b);
        return st;
    };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MS_ERR_CUDA);

    // Union tables.
    std::vector<int32_t> idx(8ULL * T, 0);
    std::vector<double> coef;
    std::vector<float> mcoef;
    if (precision == MS_PRECISION_MIXED) mcoef.resize(24ULL * T);
    else coef.resize(24ULL * T);
    std::vector<double> aux(4ULL * T), thick(T), shear(T), mass(N), pos(3ULL * N), vel(3ULL * N, 0.0);
    std::vector<unsigned char> fixed(N);
    std::vector<int> node_inst(N), off(N + 1, 0), ent(6ULL * T);
    b->ip.resize(n);
    b->init_state.resize(n);
    bool any_nonuniform = false;
    long long nb = 0, tb = 0;
    for (int i = 0; i < n; ++i) {
        const ms_batch_instance& in = inst[i];
        const ms_mesh_desc& d = in.mesh;
        const int Ni = d.num_nodes, Ti = d.num_tris;
        InstParams& q = b->ip[i];
        q.dt = in.timestep;
        q.damping1 = in.damping_factor_1;
        q.damping2 = in.damping_factor_2;
        q.rho_hh = in.params.ref_density * in.params.min_ref_thickness * in.params.min_ref_thickness;
        q.force_limit = 50000.0 * in.params.char_force_scale;
        q.nu = in.params.def_poisson_ratio;
        q.gamma = in.params.bend_stiffening_scale_factor;
        q.h = d.ref_thickness[0];
        q.mu = d.ref_shear_modulus[0];
        dev::material_coefs(q.h, q.mu, q.nu, q.gamma, q.ks, q.kb, q.igmh);
        q.uniform_hmu = 1;
        for (int t = 1; t < Ti && q.uniform_hmu; ++t)
            q.uniform_hmu = d.ref_thickness[t] == q.h && d.ref_shear_modulus[t] == q.mu;
        any_nonuniform = any_nonuniform || !q.uniform_hmu;
        q.char_force = in.params.char_force_scale;
        q.char_speed = in.params.char_speed_scale;
        q.force_thresh = in.params.force_to_char_force_ratio_equil_threshold;
        q.speed_thresh = in.params.speed_to_char_speed_ratio_equil_threshold;
        q.spacing = in.dial_factors_to_hold_at_spacing;
        q.lam_final = in.abar_info[1];
        q.nu_ot = in.abar_info[2];
        q.steps_per_phase = in.timesteps_per_dial_phase;
        q.steps_between_checks = in.timesteps_between_equil_checks;
        q.node_begin = (int)nb;
        q.node_end = (int)(nb + Ni);
        q.stop_at_final = in.stop_at_final_equilibrium ? 1 : 0;
        b->init_state[i] = initial_state(in);
        for (int t = 0; t < Ti; ++t) {
            const long long u = tb + t;
            for (int k = 0; k < 6; ++k) idx[8ULL * u + k] = (int32_t)(nb + d.patch_ids[6LL * t + k]);
            idx[8ULL * u + 7] = i;
            const double* w = d.deriv_coeffs + 24LL * t;
            if (precision == MS_PRECISION_MIXED) {
                for (int k = 0; k < 24; ++k) mcoef[24ULL * u + k] = (float)w[k];
            } else {
                std::memcpy(&coef[24ULL * u], w, 24 * sizeof(double));
            }
            const double ang = in.abar_info[3LL * t], c = std::cos(ang), s = std::sin(ang);
            aux[4ULL * u] = d.ref_area[t];
            aux[4ULL * u + 1] = c * c;
            aux[4ULL * u + 2] = s * s;
            aux[4ULL * u + 3] = c * s;
            thick[u] = d.ref_thickness[t];
            shear[u] = d.ref_shear_modulus[t];
            for (int k = 0; k < 6; ++k) off[nb + d.patch_ids[6LL * t + k] + 1] += 1;
        }
        for (int k = 0; k < Ni; ++k) {
            node_inst[nb + k] = i;
            mass[nb + k] = d.node_mass[k];
            fixed[nb + k] = d.is_constrained[k];
            for (int c = 0; c < 3; ++c) {
                pos[(size_t)c * N + nb + k] = in.dofs[(size_t)c * Ni + k];
                if (in.velocities) vel[(size_t)c * N + nb + k] = in.velocities[(size_t)c * Ni + k];
            }
        }
        nb += Ni;
        tb += Ti;
    }
    for (long long k = 0; k < N; ++k) off[k + 1] += off[k];
    {
        std::vector<int> fill(off.begin(), off.end() - 1);
        for (long long t = 0; t < T; ++t)
            for (int k = 0; k < 6; ++k) ent[fill[idx[8ULL * t + k]]++] = (int)(6 * t + k);
    }

    DevMesh& m = b->m;
    DevState& s = b->s;
    ClusterPlan& p = b->p;
    m.N = (int)N;
    m.T = (int)T;
    ms_status st;
    int4* d_idx;
    double4* d_aux;
    double *d_mass, *d_thick = nullptr, *d_shear = nullptr;
    unsigned char* d_fixed;
    int *d_off, *d_ent;
    if ((st = balloc(b, &d_idx, 2ULL * T)) || (st = balloc(b, &d_aux, T))) return bail(st);
    if (cudaMemcpy(d_idx, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(bcuda(b, cudaGetLastError(), "upload"));
    std::vector<int> soff, sent;
    build_sell((int)N, off.data(), ent.data(), soff, sent);
    int *d_soff, *d_sent;
    if ((st = bupload(b, &d_mass, mass)) || (st = bupload(b, &d_fixed, fixed)) || (st = bupload(b, &d_off, off)) ||
        (st = bupload(b, &d_ent, ent)) || (st = bupload(b, &b->d_node_inst, node_inst)) ||
        (st = bupload(b, &d_soff, soff)) || (st = bupload(b, &d_sent, sent)))
        return bail(st);
    m.sell_off = d_soff;
    m.sell_ent = d_sent;
    if (any_nonuniform && ((st = bupload(b, &d_thick, thick)) || (st = bupload(b, &d_shear, shear))))
        return bail(st);
    if (precision == MS_PRECISION_MIXED) {
        float *d_mc, *d_cf;
        if ((st = bupload(b, &d_mc, mcoef)) || (st = balloc(b, &d_cf, 6ULL * kMixedSlot * T))) return bail(st);
        p.coef_aos_f = d_mc;
        m.contrib_f = d_cf;
    } else {
        double *d_coef, *d_contrib;
        if ((st = bupload(b, &d_coef, coef)) || (st = balloc(b, &d_contrib, 18ULL * T))) return bail(st);
        p.coef_aos = d_coef;
        s.contrib = d_contrib;
    }
    p.tri_idx = d_idx;
    p.tri_aux = d_aux;
    p.lce_uniform = 1;
    // Tile records for the bulk-copy tile kernel (the default schedule on
    // unions too small for the node-tiled one).
    {
        const int mixed = precision == MS_PRECISION_MIXED;
        int blocks = 0;
        cudaError_t ea = mixed ? cudaFuncSetAttribute(k_batch_tri_tiles<true>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      2 * tiles::TileLayout<true>::bytes)
                               : cudaFuncSetAttribute(k_batch_tri_tiles<false>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      2 * tiles::TileLayout<false>::bytes);
        if (ea == cudaSuccess)
            ea = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_batch_tri_tiles<true>, kTile,
                                                                       2 * tiles::TileLayout<true>::bytes)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_batch_tri_tiles<false>, kTile,
                                                                       2 * tiles::TileLayout<false>::bytes);
        if (ea == cudaSuccess && blocks > 0) {
            const size_t rec = mixed ? tiles::TileLayout<true>::bytes : tiles::TileLayout<false>::bytes;
            const long long ntiles = (T + kTile - 1) / kTile;
            std::vector<unsigned char> buf(rec * ntiles, 0);
            const size_t ids_b = 6 * kTile * 4, coef_b = 24 * kTile * (mixed ? 4 : 8);
            for (long long t = 0; t < T; ++t) {
                const long long tile = t / kTile, li = t % kTile;
                unsigned char* r = buf.data() + rec * tile;
                int32_t* ids = reinterpret_cast<int32_t*>(r);
                double* ax = reinterpret_cast<double*>(r + ids_b + coef_b);
                for (int k = 0; k < 6; ++k) ids[k * kTile + li] = idx[8ULL * t + k];
                if (mixed) {
                    float* c = reinterpret_cast<float*>(r + ids_b);
                    for (int k = 0; k < 24; ++k) c[k * kTile + li] = mcoef[24ULL * t + k];
                } else {
                    double* c = reinterpret_cast<double*>(r + ids_b);
                    for (int k = 0; k < 24; ++k) c[k * kTile + li] = coef[24ULL * t + k];
                }
                for (int k = 0; k < 4; ++k) ax[k * kTile + li] = aux[4ULL * t + k];
            }
            unsigned char* d_tiles;
            if ((st = bupload(b, &d_tiles, buf))) return bail(st);
            if (mixed) p.tiles_f = d_tiles;
            else p.tiles = d_tiles;
            int dev = 0, sms = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            b->tile_grid = sms * blocks;
        } else {
            cudaGetLastError();
            b->tile_grid = 0;
        }
    }
    {
        std::vector<int> tri_inst(T);
        for (long long t = 0; t < T; ++t) tri_inst[t] = idx[8ULL * t + 7];
        if ((st = bupload(b, &b->d_tri_inst, tri_inst)) || (st = balloc(b, &b->d_err, 1))) return bail(st);
        if (cudaMemset(b->d_err, 0, sizeof(int)) != cudaSuccess) return bail(MS_ERR_CUDA);
    }
    // Node-tiled one-kernel step over the union (node_tile_plan.cu).
    {
        const int mixed = precision == MS_PRECISION_MIXED;
        std::vector<int> patch6(6ULL * T);
        for (long long t = 0; t < T; ++t)
            for (int k = 0; k < 6; ++k) patch6[6ULL * t + k] = idx[8ULL * t + k];
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        auto blocks_for = [&](size_t smem) { return batch_node_tile_blocks(mixed, smem); };
        NodeTileLayout L;
        std::string err;
        int NT = 0, blocks = 0;
        auto smem_for = [&](const NodeTileLayout& lay, int nodes) { return node_tile_smem(lay.stride, nodes, mixed); };
        if (!choose_node_tiles(patch6.data(), (int)N, (int)T, mixed, sms, mixed ? MSB_NT_MINB_MIXED : MSB_NT_MINB,
                               mixed ? 1008 : 1100, 256, off, ent, smem_for, blocks_for, L, NT, blocks, err))
            return bail(bfail(b, MS_ERR_INVALID_ARGUMENT, err));
        if (blocks > 0) {
            if ((st = plan_from_layout(b, L, NT, blocks, b->ntp, b->nt_allocs))) return bail(st);
            b->nt_blocks = blocks;
            b->have_nt = true;
        }
        // The one-kernel step once every block has a tile of its own
        // (measured fastest on B200 for the single-mesh step), else the
        // tile kernel, else the per-triangle kernel.
        b->sched = (b->have_nt && b->ntp.ntiles >= b->ntp.grid) ? kSchedNodeTiles
                   : b->tile_grid > 0                         ? kSchedTiles
                                                              : kSchedAos;
    }
    m.mass = d_mass;
    m.fixed = d_fixed;
    m.inc_off = d_off;
    m.inc_ent = d_ent;
    m.thick = d_thick;
    m.shear = d_shear;
    for (int k = 0; k < 2; ++k) {
        if ((st = balloc(b, &s.pos[k], 3ULL * N)) || (st = balloc(b, &s.vel[k], 3ULL * N))) return bail(st);
    }
    if (cudaMemcpy(s.pos[0], pos.data(), sizeof(double) * pos.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s.vel[0], vel.data(), sizeof(double) * vel.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s.pos[1], pos.data(), sizeof(double) * pos.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s.vel[1], vel.data(), sizeof(double) * vel.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(bcuda(b, cudaGetLastError(), "upload state"));
    if ((st = balloc(b, &b->d_fnorm, N)) || (st = balloc(b, &b->d_vnorm, N)) || (st = bupload(b, &b->d_ip, b->ip)) ||
        (st = bupload(b, &b->d_is, b->init_state)))
        return bail(st);
    if (cudaMallocHost(&b->h_is, sizeof(InstState) * n) != cudaSuccess) return bail(MS_ERR_OUT_OF_MEMORY);
    std::memcpy(b->h_is, b->init_state.data(), sizeof(InstState) * n);
    *out = b;
    return MS_OK;
}

void ms_batch_destroy(ms_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    clear_graphs(b);
    for (void* q : b->allocs) cudaFree(q);
    for (void* q : b->nt_allocs) cudaFree(q);
    if (b->h_is) cudaFreeHost(b->h_is);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* ms_batch_last_error(const ms_batch* b) { return b ? b->last_error.c_str() : "null batch"; }

ms_status ms_batch_run(ms_batch* b, int64_t max_steps, int64_t* steps_done) {
    if (!b || max_steps < 0) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    int64_t done = 0;
    MB_TRY(fetch_states(b));
    while (done < max_steps && !all_frozen(b)) {
        const int len = (int)std::min<int64_t>(b->chunk, max_steps - done);
        MB_TRY(run_graph(b, len, b->parity, b->sched));
        b->parity ^= len & 1;
        done += len;
        MB_TRY(fetch_states(b));
    }
    if (steps_done) *steps_done = done;
    return MS_OK;
}

ms_status ms_batch_status(ms_batch* b, int32_t i, ms_batch_inst_status* out) {
    if (!b || !out || i < 0 || i >= b->n_inst) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    MB_TRY(fetch_states(b));
    const InstState& st = b->h_is[i];
    const InstParams& q = b->ip[i];
    out->status = st.status;
    out->equilibria = st.equilibria;
    out->stepcount = st.stepcount;
    out->dial_factor = st.dial_factor;
    out->last_equil_dial = st.last_equil_dial;
    out->sim_time = st.time;
    out->max_force_ratio = st.max_force / q.char_force;
    out->max_speed_ratio = st.max_speed / q.char_speed;
    out->max_force_node = st.max_force_node;
    out->max_speed_node = st.max_speed_node;
    out->offending_dof = st.guard_key == ~0ULL ? -1 : (int64_t)st.guard_key;
    return MS_OK;
}

ms_status ms_batch_download_dofs(ms_batch* b, int32_t i, double* dofs, double* vel) {
    if (!b || i < 0 || i >= b->n_inst) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    MB_TRY(fetch_states(b));
    const InstState& st = b->h_is[i];
    const int buf = st.frozen_parity >= 0 ? st.frozen_parity : b->parity;
    const InstParams& q = b->ip[i];
    const size_t Ni = (size_t)(q.node_end - q.node_begin), N = (size_t)b->m.N;
    for (int c = 0; c < 3; ++c) {
        if (dofs)
            MB_CUDA(b, cudaMemcpy(dofs + c * Ni, b->s.pos[buf] + c * N + q.node_begin, Ni * sizeof(double),
                                  cudaMemcpyDeviceToHost));
        if (vel)
            MB_CUDA(b, cudaMemcpy(vel + c * Ni, b->s.vel[buf] + c * N + q.node_begin, Ni * sizeof(double),
                                  cudaMemcpyDeviceToHost));
    }
    return MS_OK;
}

ms_status ms_batch_upload_dofs(ms_batch* b, int32_t i, const double* dofs, const double* vel) {
    if (!b || !dofs || i < 0 || i >= b->n_inst) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    MB_CUDA(b, cudaStreamSynchronize(b->stream));
    const InstParams& q = b->ip[i];
    const size_t Ni = (size_t)(q.node_end - q.node_begin), N = (size_t)b->m.N;
    std::vector<double> zero(vel ? 0 : Ni, 0.0);
    for (int k = 0; k < 2; ++k)
        for (int c = 0; c < 3; ++c) {
            MB_CUDA(b, cudaMemcpy(b->s.pos[k] + c * N + q.node_begin, dofs + c * Ni, Ni * sizeof(double),
                                  cudaMemcpyHostToDevice));
            MB_CUDA(b, cudaMemcpy(b->s.vel[k] + c * N + q.node_begin, vel ? vel + c * Ni : zero.data(),
                                  Ni * sizeof(double), cudaMemcpyHostToDevice));
        }
    MB_CUDA(b, cudaMemcpy(b->d_is + i, &b->init_state[i], sizeof(InstState), cudaMemcpyHostToDevice));
    return MS_OK;
}

ms_status ms_batch_set_start(ms_batch* b, int32_t i, double dial_factor, int32_t waiting) {
    if (!b || i < 0 || i >= b->n_inst || !(dial_factor >= 0.0) || dial_factor > 1.0) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    MB_CUDA(b, cudaStreamSynchronize(b->stream));
    const InstParams& q = b->ip[i];
    InstState st = b->init_state[i];
    st.dial_factor = st.last_equil_dial = dial_factor;
    if (waiting) {
        // As main.cpp:293-304 leaves a finished dial phase: waiting, the
        // check counter at zero, the second damping factor, and the
        // programmed metric held at this dial factor.
        st.status = INST_WAITING;
        st.k_phase = q.steps_per_phase;
        st.tsc = 0;
        st.damping = q.damping2;
        st.cur_dial = dial_factor;
        st.cur_lam = (1.0 - dial_factor) * 1.0 + dial_factor * q.lam_final;
        st.cur_pw = std::pow(st.cur_lam, -2.0 * q.nu_ot);
    } else {
        st.k_phase = static_cast<long long>(std::fmod(dial_factor, q.spacing) * static_cast<double>(q.steps_per_phase));
    }
    b->init_state[i] = st;
    MB_CUDA(b, cudaMemcpy(b->d_is + i, &st, sizeof(InstState), cudaMemcpyHostToDevice));
    return MS_OK;
}

ms_status ms_batch_set_schedule(ms_batch* b, const ms_batch_schedule* s) {
    if (!b || !s) return MS_ERR_INVALID_ARGUMENT;
    if (s->chunk_steps <= 0 || s->chunk_steps % 2 || s->chunk_steps > 1024)
        return bfail(b, MS_ERR_INVALID_ARGUMENT, "chunk_steps must be even, 2..1024");
    for (int k = 0; k < kNumScheds; ++k)
        if (kScheds[k].tri_block == s->tri_block &&
            (kScheds[k].node_block == s->node_block || s->tri_block < 0) && (s->tri_block != 0 || b->tile_grid > 0) &&
            (s->tri_block >= 0 || b->have_nt)) {
            b->sched = k;
            b->chunk = s->chunk_steps;
            return MS_OK;
        }
    return bfail(b, MS_ERR_UNSUPPORTED, "no built-in schedule with these block sizes");
}

ms_status ms_batch_get_schedule(const ms_batch* b, ms_batch_schedule* s) {
    if (!b || !s) return MS_ERR_INVALID_ARGUMENT;
    s->tri_block = kScheds[b->sched].tri_block;
    s->node_block = kScheds[b->sched].node_block;
    s->chunk_steps = b->chunk;
    s->nodes_per_tile = b->have_nt ? b->ntp.nodes : 0;
    s->blocks_per_sm = b->have_nt ? b->nt_blocks : 0;
    return MS_OK;
}

ms_status ms_batch_autotune(ms_batch* b, int32_t steps, ms_batch_schedule* chosen, double* best_ms) {
    if (!b || steps <= 0) return MS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(b->device);
    steps += steps & 1;
    const size_t N = (size_t)b->m.N, n = (size_t)b->n_inst;
    double *save_pos, *save_vel;
    InstState* save_is;
    MB_CUDA(b, cudaMalloc(&save_pos, 3 * N * sizeof(double)));
    cudaError_t e1 = cudaMalloc(&save_vel, 3 * N * sizeof(double));
    cudaError_t e2 = cudaMalloc(&save_is, n * sizeof(InstState));
    auto release = [&]() {
        cudaFree(save_pos);
        if (e1 == cudaSuccess) cudaFree(save_vel);
        if (e2 == cudaSuccess) cudaFree(save_is);
    };
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        release();
        return bfail(b, MS_ERR_OUT_OF_MEMORY, "autotune: no room to save the state");
    }
    const int p0 = b->parity;
    const int keep_sched = b->sched;
    cudaStream_t st = b->stream;
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    double best = 1e300;
    int best_k = keep_sched;
    ms_status rc = MS_OK;
    auto copy_state = [&](bool save) -> cudaError_t {
        cudaError_t e;
        if (save) {
            if ((e = cudaMemcpyAsync(save_pos, b->s.pos[p0], 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st)))
                return e;
            if ((e = cudaMemcpyAsync(save_vel, b->s.vel[p0], 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st)))
                return e;
            return cudaMemcpyAsync(save_is, b->d_is, n * sizeof(InstState), cudaMemcpyDeviceToDevice, st);
        }
        if ((e = cudaMemcpyAsync(b->s.pos[p0], save_pos, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st)))
            return e;
        if ((e = cudaMemcpyAsync(b->s.vel[p0], save_vel, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st)))
            return e;
        return cudaMemcpyAsync(b->d_is, save_is, n * sizeof(InstState), cudaMemcpyDeviceToDevice, st);
    };
    if (copy_state(true) != cudaSuccess) rc = bcuda(b, cudaGetLastError(), "autotune save");
    const int mixed = b->precision == MS_PRECISION_MIXED;
    std::string report;
    // ms per step of schedule k from the saved state: one untimed pass
    // (graph instantiation, caches), then the timed one; < 0 on error (rc).
    auto time_sched = [&](int k) -> double {
        if (kScheds[k].tri_block < 0)  // the launch's shared memory is the current plan's
            batch_node_tile_blocks(mixed, node_tile_smem(b->ntp.stride, b->ntp.nodes, mixed));
        double t = -1.0;
        for (int rep = 0; rep < 2 && rc == MS_OK; ++rep) {
            if (copy_state(false) != cudaSuccess) {
                rc = bcuda(b, cudaGetLastError(), "autotune restore");
                break;
            }
            cudaEventRecord(ev0, st);
            rc = run_graph(b, steps, p0, k);
            cudaEventRecord(ev1, st);
            if (rc != MS_OK) break;
            if (cudaEventSynchronize(ev1) != cudaSuccess) {
                rc = bcuda(b, cudaGetLastError(), "autotune");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            if (rep == 1) t = ms / steps;
        }
        return t;
    };
    double nt_ms = -1.0;
    for (int k = 0; k < kNumScheds && rc == MS_OK; ++k) {
        if (kScheds[k].tri_block == 0 && b->tile_grid == 0) continue;
        if (kScheds[k].tri_block < 0 && !b->have_nt) continue;
        const double t = time_sched(k);
        if (t < 0) break;
        char line[160];
        std::snprintf(line, sizeof line, "schedule tri_block %d node_block %d%s: %.4f ms/step\n",
                      kScheds[k].tri_block, kScheds[k].node_block,
                      k == kSchedNodeTiles ? (" (" + std::to_string(b->ntp.nodes) + "-node tiles, " +
                                              std::to_string(b->nt_blocks) + " blocks/SM)").c_str()
                                           : "",
                      t);
        report += line;
        if (k == kSchedNodeTiles) nt_ms = t;
        if (t < best) {
            best = t;
            best_k = k;
        }
    }
    // Tile size and resident blocks per SM of the node-tiled plan: rebuild
    // it at smaller and larger tiles, and at larger tiles with one block per
    // SM fewer, time each, keep the fastest (the plans give the same bits).
    if (rc == MS_OK && nt_ms > 0) {
        const int N = b->m.N, T = b->m.T;
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        std::vector<int4> idx(2ULL * T);
        std::vector<int> patch6(6ULL * T), off(N + 1), ent(6ULL * T);
        if (cudaMemcpy(idx.data(), b->p.tri_idx, sizeof(int4) * idx.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(off.data(), b->m.inc_off, sizeof(int) * off.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(ent.data(), b->m.inc_ent, sizeof(int) * ent.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = bcuda(b, cudaGetLastError(), "autotune: incidence download");
        for (long long t = 0; t < T && rc == MS_OK; ++t) {
            const int4 a = idx[2 * t], c = idx[2 * t + 1];
            const int id[6] = {a.x, a.y, a.z, a.w, c.x, c.y};
            for (int k = 0; k < 6; ++k) patch6[6 * t + k] = id[k];
        }
        const int nt0 = b->ntp.nodes, b0 = b->nt_blocks;
        const int cand[3][2] = {{nt0 * 7 / 10, b0}, {nt0 * 14 / 10, b0}, {nt0 * 2, b0 - 1}};
        for (const auto& cd : cand) {
            if (rc != MS_OK) break;
            const int nt = std::max(256, std::min(cd[0], kNtMaxNodes)), nb = cd[1];
            if (nb < 1 || nt == b->ntp.nodes) continue;
            NodeTileLayout L;
            std::string err;
            if (!node_tile_layout(patch6.data(), N, T, nt, mixed, off, ent, L, err)) continue;
            if (L.K < sms * nb || batch_node_tile_blocks(mixed, node_tile_smem(L.stride, nt, mixed)) < nb) continue;
            NodeTilePlan q;
            std::vector<void*> al;
            const ms_status s2 = plan_from_layout(b, L, nt, nb, q, al);
            if (s2 != MS_OK) {  // no room for a second plan: keep the current one
                for (void* x : al) cudaFree(x);
                cudaGetLastError();
                if (s2 != MS_ERR_OUT_OF_MEMORY) rc = s2;
                continue;
            }
            std::swap(b->ntp, q);
            clear_graphs(b);
            const double t = time_sched(kSchedNodeTiles);
            char line[160];
            std::snprintf(line, sizeof line, "node-tiled plan %d-node tiles, %d blocks/SM: %.4f ms/step\n", nt, nb, t);
            report += line;
            if (t > 0 && t < nt_ms) {
                for (void* x : b->nt_allocs) cudaFree(x);
                b->nt_allocs.swap(al);
                b->nt_blocks = nb;
                nt_ms = t;
                if (t < best) {
                    best = t;
                    best_k = kSchedNodeTiles;
                }
            } else {
                std::swap(b->ntp, q);
                clear_graphs(b);
                for (void* x : al) cudaFree(x);
            }
        }
        batch_node_tile_blocks(mixed, node_tile_smem(b->ntp.stride, b->ntp.nodes, mixed));
    }
    if (copy_state(false) != cudaSuccess && rc == MS_OK) rc = bcuda(b, cudaGetLastError(), "autotune restore");
    cudaStreamSynchronize(st);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    release();
    b->parity = p0;
    clear_graphs(b);
    if (rc != MS_OK) {
        b->sched = keep_sched;
        return rc;
    }
    b->sched = best_k;
    b->tune_report = report;
    if (chosen) ms_batch_get_schedule(b, chosen);
    if (best_ms) *best_ms = best;
    return MS_OK;
}

int32_t ms_batch_autotune_report(const ms_batch* b, char* buf, int32_t len) {
    if (!b) return -1;
    const int32_t n = (int32_t)b->tune_report.size();
    if (buf && len > 0) {
        const int32_t k = std::min(n, len - 1);
        std::memcpy(buf, b->tune_report.data(), (size_t)k);
        buf[k] = 0;
    }
    return n;
}

ms_status ms_batch_info(const ms_batch* b, int64_t* num_nodes, int64_t* num_tris, int32_t* n_instances) {
    if (!b) return MS_ERR_INVALID_ARGUMENT;
    if (num_nodes) *num_nodes = b->m.N;
    if (num_tris) *num_tris = b->m.T;
    if (n_instances) *n_instances = b->n_inst;
    return MS_OK;
}

void* ms_batch_stream(ms_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"
