// Node-tiled step with warp-specialised roles (ms_set_step_path 4): the same
// chunk records and the same per-node summation order as the node-tiled
// kernel (node_tiles.cu), with the triangle arithmetic and the node sums
// running at the same time in different warpgroups instead of in turn.
//
// One persistent block of three warpgroups per SM walks the block's chunks
// (tiles blockIdx.x, then every gridDim.x-th; each tile's chunks in order):
//
//   math warpgroups 0 and 1 take the block's even and odd chunks.  Each has
//   its own table buffer: its thread 0 copies a chunk's record in with two
//   cp.async.bulk (the tables into the buffer, the node section into one of
//   eight node-section slots; completion counted in bytes on the group's
//   mbarrier), and starts the copy of the group's next chunk as soon as every
//   thread holds its triangle's tables in registers.  A thread computes one
//   triangle (tile_tri, the arithmetic every path shares), waits until the
//   aggregation group has released the group's staging area, stages its 18
//   contributions there field-major and arrives on the group's stage_full
//   barrier.
//
//   the aggregation warpgroup takes the chunks in order: it waits for a
//   chunk's staging area, adds the chunk's runs to the tile's per-node
//   accumulators in shared memory (one thread per run, a run being one
//   node's entries in ascending triangle order), releases the staging area,
//   and finishes a node (damping, constraints, equilibrium maxima, force
//   guard, symplectic Euler; node_core) once the run that the plan marks as
//   its last is added: the node's state is loaded into registers then, and
//   node_core runs after the next chunk's runs, so the load latency hides
//   behind that work.  Chunks are added in order, so each node's force is
//   the sum of its contributions in ascending triangle order from zero --
//   the order, and so the bits, of every other path.
//
// So the triangle arithmetic of the next two chunks overlaps the sums and
// node updates of the current one, and the node updates are spread over the
// tile's chunks instead of forming a phase of their own.
//
// Every wait is bounded (about a second of SM clock).  A warpgroup decides
// together whether to go on (a barrier with an AND reduction), so no thread
// is left at a named barrier; on a timeout the kernel records
// MS_ERR_TIMEOUT, lets its own copies in flight land (bounded) and returns.
#include <algorithm>
#include <climits>

#include "internal.cuh"
#include "step_common.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace {

using namespace stepdev;
using namespace tiles;

constexpr int kPipeThreads = 384;
constexpr int kNsSlots = 8;   // node-section slots: a chunk's slot is refilled 8 chunks later
constexpr int kAggBar = 3;    // named barrier of the aggregation group (1, 2: the math groups)
constexpr int kDefer = 2;     // final runs per aggregation thread and chunk whose node finish is deferred

// Shared memory: two table buffers, two staging areas, the node-section
// slots, the tile's per-node accumulators.
template <bool MIXED>
struct PipeSmem {
    using R = typename tridev::Real<MIXED>::T;
    static constexpr size_t tables = TileLayout<MIXED>::bytes;
    static constexpr size_t stage = (size_t)kTile * 18 * sizeof(R);
    static_assert(tables % 128 == 0 && stage % 128 == 0, "buffers stay 128-byte aligned");
    __host__ __device__ static size_t ns_cap(size_t stride) { return stride - tables; }
    __host__ __device__ static size_t bytes(size_t stride, int nodes) {
        return 2 * tables + 2 * stage + kNsSlots * ns_cap(stride) + 24 * (size_t)nodes;
    }
};

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
// True on every thread of a 128-thread group iff `ok` holds on all of them.
__device__ __forceinline__ bool group_all(bool ok, int id) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, p;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.and.pred p, %2, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)ok), "r"(id)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// The block's chunks in order: tiles blockIdx.x, then every gridDim.x-th,
// each tile's chunks in turn (a tile has at least one chunk).
struct Cursor {
    int tile, c, cend;
    __device__ __forceinline__ void start(const NodeTilePlan& q) {
        tile = blockIdx.x;
        c = cend = 0;
        if (tile < q.ntiles) {
            c = __ldg(q.tile_chunk + tile);
            cend = __ldg(q.tile_chunk + tile + 1);
        }
    }
    __device__ __forceinline__ bool valid(const NodeTilePlan& q) const { return tile < q.ntiles; }
    __device__ __forceinline__ void next(const NodeTilePlan& q) {
        if (++c < cend) return;
        tile += gridDim.x;
        if (tile < q.ntiles) {
            c = __ldg(q.tile_chunk + tile);
            cend = __ldg(q.tile_chunk + tile + 1);
        }
    }
};

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kPipeThreads, 1)
    k_node_pipe(const DevMesh m, const ClusterPlan p, const NodeTilePlan q, const DevState s, const StepScalars sc) {
    using R = typename tridev::Real<MIXED>::T;
    using L = TileLayout<MIXED>;
    using SM = PipeSmem<MIXED>;
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform over the grid
    extern __shared__ __align__(128) unsigned char pipe_smem[];
    __shared__ uint64_t full[2], stage_full[2], stage_free[2];
    const size_t ns_cap = SM::ns_cap(q.stride);
    unsigned char* tables = pipe_smem;
    unsigned char* stages = pipe_smem + 2 * SM::tables;
    unsigned char* nsec = stages + 2 * SM::stage;
    double* acc = reinterpret_cast<double*>(nsec + kNsSlots * ns_cap);
    const int tid = threadIdx.x, wg = tid >> 7, i = tid & 127;
    for (int j = tid; j < 3 * q.nodes; j += kPipeThreads) acc[j] = 0.0;
    if (tid == 0) {
        for (int w = 0; w < 2; ++w) {
            mbar_init(&full[w], 1);
            mbar_init(&stage_full[w], 128);
            mbar_init(&stage_free[w], 128);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (wg < 2) {
        // ---- math group w: chunks w, w + 2, w + 4, ... of the block -------
        const int w = wg;
        const double* pos = pos_buf(s, sc.parity);
        double dial = 0.0, lam = 0.0, pw = 0.0;
        if (DIAL == DIAL_LCE) {
            dial = s.dials[3 * gstep];
            lam = s.dials[3 * gstep + 1];
            pw = s.dials[3 * gstep + 2];
        }
        // The triangle id of a slot is needed only for per-triangle
        // material, per-triangle LCE fields or programmed tensors read from
        // arrays.
        const bool need_t = DIAL != DIAL_LCE || !p.lce_uniform || !m.uniform_hmu;
        unsigned char* tb = tables + w * SM::tables;
        R* stage = reinterpret_cast<R*>(stages + w * SM::stage);
        // Thread 0: chunk c (the block's g-th) into this group's table buffer
        // and node-section slot g % kNsSlots.  That slot last held chunk
        // g - kNsSlots, whose runs the aggregation group finished before it
        // released this group's staging area for chunk g - 4.
        auto fetch = [&](int c, int g) {
            const unsigned char* src = q.rec + (size_t)c * q.stride;
            const uint32_t nb = __ldg(q.chunk_bytes + c) - (uint32_t)SM::tables;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&full[w])),
                         "r"((uint32_t)SM::tables + nb)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(tb)),
                "l"(src), "r"((uint32_t)SM::tables), "r"(smem_addr(&full[w]))
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(nsec + (size_t)(g % kNsSlots) * ns_cap)),
                "l"(src + SM::tables), "r"(nb), "r"(smem_addr(&full[w]))
                : "memory");
        };
        Cursor cur;
        cur.start(q);
        int g = 0;
        if (w == 1) {
            cur.next(q);
            g = 1;
        }
        bool pending = cur.valid(q);  // a copy of this group is in flight
        if (i == 0 && pending) fetch(cur.c, g);
        int k = 0;  // chunks of this group so far
        while (cur.valid(q)) {
            if (!group_all(bar_wait(&full[w], k & 1), 1 + w)) {
                if (i == 0) atomicCAS(&s.err->flag, 0, 5);  // MS_ERR_TIMEOUT
                break;
            }
            pending = false;
            const unsigned char* ns = nsec + (size_t)(g % kNsSlots) * ns_cap;
            const int ntri = reinterpret_cast<const int*>(ns)[2];
            const int* sid = reinterpret_cast<const int*>(tb);
            const R* scoef = reinterpret_cast<const R*>(tb + L::ids);
            const double* saux = reinterpret_cast<const double*>(tb + L::ids + L::coef);
            int ids[6];
            R cf[24];
#pragma unroll
            for (int j = 0; j < 6; ++j) ids[j] = sid[j * kTile + i];
#pragma unroll
            for (int j = 0; j < 24; ++j) cf[j] = scoef[j * kTile + i];
            const double area = saux[i], c2 = saux[kTile + i], s2 = saux[2 * kTile + i], cs = saux[3 * kTile + i];
            const bool live = i < ntri;
            const int t = (need_t && live) ? __ldg(q.chunk_tri + (size_t)cur.c * kTile + i) : 0;
            // Order the table reads before the bulk copy that refills the
            // buffer.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            group_sync(1 + w);
            Cursor nx = cur;
            nx.next(q);
            nx.next(q);
            if (nx.valid(q)) {
                if (i == 0) fetch(nx.c, g + 2);
                pending = true;
            }
            R f[18];
#pragma unroll
            for (int j = 0; j < 18; ++j) f[j] = R(0);
            if (live) tile_tri<DIAL, MIXED>(m, p, pos, dial, lam, pw, t, ids, cf, area, c2, s2, cs, f);
            // The staging area is free once the aggregation group has added
            // this group's previous chunk.
            if (k > 0 && !group_all(bar_wait(&stage_free[w], (k - 1) & 1), 1 + w)) {
                if (i == 0) atomicCAS(&s.err->flag, 0, 5);
                ++k;  // the copy in flight completes phase k + 1 of `full`
                break;
            }
#pragma unroll
            for (int j = 0; j < 18; ++j) stage[j * kTile + i] = f[j];
            mbar_arrive(&stage_full[w]);
            cur = nx;
            g += 2;
            ++k;
        }
        // Leave no copy of this group in flight.
        if (i == 0 && pending) bar_wait(&full[w], k & 1);
    } else {
        // ---- aggregation group: every chunk of the block, in order --------
        // A node whose last run is one of the thread's first kDefer runs of
        // a chunk is finished one chunk later: its state is loaded into
        // registers as soon as its force is complete, and node_core runs
        // after the next chunk's runs, so the loads take no round trip of
        // their own.  Later final runs of a chunk (more than kDefer x 128
        // runs) are finished at once.
        double fmax = -1.0, vmax = -1.0;
        int fnode = INT_MAX, vnode = INT_MAX;
        int dn[kDefer];
        double dF[kDefer][3];
        NodeIn din[kDefer];
#pragma unroll
        for (int k = 0; k < kDefer; ++k) dn[k] = -1;
        auto add_run = [&](const R* stage, const unsigned short* re, const unsigned short* en, int r, int j,
                           double& a0, double& a1, double& a2) {
            int e = r ? re[r - 1] : 0;
            const int e1 = re[r];
            a0 = acc[3 * j];
            a1 = acc[3 * j + 1];
            a2 = acc[3 * j + 2];
            for (; e < e1; ++e) {
                const R* v = stage + en[e];
                a0 += (double)v[0];
                a1 += (double)v[kTile];
                a2 += (double)v[2 * kTile];
            }
        };
        Cursor cur;
        cur.start(q);
        bool aborted = false;
        for (int g = 0; cur.valid(q); ++g, cur.next(q)) {
            const int w = g & 1;
            if (!group_all(bar_wait(&stage_full[w], (g >> 1) & 1), kAggBar)) {
                if (i == 0) atomicCAS(&s.err->flag, 0, 5);
                aborted = true;
                break;
            }
            const R* stage = reinterpret_cast<const R*>(stages + w * SM::stage);
            const unsigned char* ns = nsec + (size_t)(g % kNsSlots) * ns_cap;
            const int nruns = reinterpret_cast<const int*>(ns)[0];
            const unsigned short* rn = reinterpret_cast<const unsigned short*>(ns + 16);
            const unsigned short* re = rn + nruns;
            const unsigned short* en = re + nruns;
            const int n0 = cur.tile * q.nodes;
            int cn[kDefer];
            double cF[kDefer][3];
            NodeIn cin[kDefer];
#pragma unroll
            for (int k = 0; k < kDefer; ++k) {
                cn[k] = -1;
                const int r = i + 128 * k;
                if (r < nruns) {
                    const unsigned u = rn[r];
                    const int j = u & ~kRunFinal;
                    double a0, a1, a2;
                    add_run(stage, re, en, r, j, a0, a1, a2);
                    if (u & kRunFinal) {
                        // The node's force is complete: clear its
                        // accumulator for the block's next tile, start
                        // loading its state, finish it after the next chunk.
                        acc[3 * j] = acc[3 * j + 1] = acc[3 * j + 2] = 0.0;
                        cn[k] = n0 + j;
                        cF[k][0] = a0;
                        cF[k][1] = a1;
                        cF[k][2] = a2;
                        cin[k] = node_load(m, s, sc, n0 + j);
                    } else {
                        acc[3 * j] = a0;
                        acc[3 * j + 1] = a1;
                        acc[3 * j + 2] = a2;
                    }
                }
            }
            for (int r = i + 128 * kDefer; r < nruns; r += 128) {
                const unsigned u = rn[r];
                const int j = u & ~kRunFinal;
                double a0, a1, a2;
                add_run(stage, re, en, r, j, a0, a1, a2);
                if (u & kRunFinal) {
                    acc[3 * j] = acc[3 * j + 1] = acc[3 * j + 2] = 0.0;
                    const int n = n0 + j;
                    node_core(m, s, sc, gstep, n, node_load(m, s, sc, n), a0, a1, a2, fmax, fnode, vmax, vnode);
                } else {
                    acc[3 * j] = a0;
                    acc[3 * j + 1] = a1;
                    acc[3 * j + 2] = a2;
                }
            }
            // This chunk's node-section slot is refilled by a bulk copy later.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&stage_free[w]);
            // The previous chunk's deferred nodes: their state has landed.
#pragma unroll
            for (int k = 0; k < kDefer; ++k) {
                if (dn[k] >= 0)
                    node_core(m, s, sc, gstep, dn[k], din[k], dF[k][0], dF[k][1], dF[k][2], fmax, fnode, vmax, vnode);
                dn[k] = cn[k];
                dF[k][0] = cF[k][0];
                dF[k][1] = cF[k][1];
                dF[k][2] = cF[k][2];
                din[k] = cin[k];
            }
            // The next chunk's runs may add to the same nodes.
            group_sync(kAggBar);
        }
        if (!aborted) {
#pragma unroll
            for (int k = 0; k < kDefer; ++k)
                if (dn[k] >= 0)
                    node_core(m, s, sc, gstep, dn[k], din[k], dF[k][0], dF[k][1], dF[k][2], fmax, fnode, vmax, vnode);
        }
        if (sc.check) {
            // Block max/argmax over the aggregation group, then the grid fold.
            __shared__ double sf[4], sv[4];
            __shared__ int sfn[4], svn[4];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double of = __shfl_down_sync(0xffffffffu, fmax, o);
                const int ofn = __shfl_down_sync(0xffffffffu, fnode, o);
                const double ov = __shfl_down_sync(0xffffffffu, vmax, o);
                const int ovn = __shfl_down_sync(0xffffffffu, vnode, o);
                eq_merge(fmax, fnode, of, ofn);
                eq_merge(vmax, vnode, ov, ovn);
            }
            const int lane = i & 31, warp = i >> 5;
            if (lane == 0) {
                sf[warp] = fmax;
                sfn[warp] = fnode;
                sv[warp] = vmax;
                svn[warp] = vnode;
            }
            group_sync(kAggBar);
            if (i == 0) {
                EqPartial r{sf[0], sv[0], sfn[0], svn[0]};
                for (int k = 1; k < 4; ++k) {
                    eq_merge(r.f, r.fn, sf[k], sfn[k]);
                    eq_merge(r.v, r.vn, sv[k], svn[k]);
                }
                s.eq_part[blockIdx.x] = r;
                __threadfence();
                const unsigned done = atomicAdd(s.eq_counter, 1u);
                if (done == gridDim.x - 1) {
                    __threadfence();
                    double F = -1.0, V = -1.0;
                    int Fn = INT_MAX, Vn = INT_MAX;
                    for (int b = 0; b < (int)gridDim.x; ++b) {
                        const volatile EqPartial* pp = s.eq_part + b;
                        eq_merge(F, Fn, pp->f, pp->fn);
                        eq_merge(V, Vn, pp->v, pp->vn);
                    }
                    s.equil->max_force = F;
                    s.equil->max_speed = V;
                    s.equil->max_force_node = Fn;
                    s.equil->max_speed_node = Vn;
                    *s.eq_counter = 0u;
                }
            }
        }
    }
}

template <int DIAL, bool MIXED>
cudaError_t launch_one(const DevMesh& m, const ClusterPlan& p, const NodeTilePlan& q, const DevState& s,
                       const StepScalars& sc, cudaStream_t st) {
    const int grid = std::min(q.ntiles, q.grid_pipe);
    if (grid <= 0) return cudaSuccess;
    k_node_pipe<DIAL, MIXED><<<grid, kPipeThreads, PipeSmem<MIXED>::bytes(q.stride, q.nodes), st>>>(m, p, q, s, sc);
    return cudaGetLastError();
}

template <int DIAL, bool MIXED>
cudaError_t prepare_one(size_t smem, int& blocks) {
    cudaError_t e =
        cudaFuncSetAttribute(k_node_pipe<DIAL, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_node_pipe<DIAL, MIXED>, kPipeThreads, smem);
    if (e != cudaSuccess) return e;
    blocks = blocks == 0 ? b : std::min(blocks, b);
    return cudaSuccess;
}

}  // namespace

size_t node_pipe_smem(size_t stride, int nodes, int mixed) {
    return mixed ? PipeSmem<true>::bytes(stride, nodes) : PipeSmem<false>::bytes(stride, nodes);
}

cudaError_t prepare_node_pipe_kernels(int mixed, size_t smem, int* blocks_per_sm) {
    int b = 0;
    cudaError_t e = mixed ? prepare_one<DIAL_LCE, true>(smem, b) : prepare_one<DIAL_LCE, false>(smem, b);
    if (e == cudaSuccess) e = mixed ? prepare_one<DIAL_ARRAYS, true>(smem, b) : prepare_one<DIAL_ARRAYS, false>(smem, b);
    *blocks_per_sm = b;
    return e;
}

cudaError_t launch_node_pipe(const DevMesh& m, const ClusterPlan& p, const NodeTilePlan& q, const DevState& s,
                             const StepScalars& sc, int dial_mode, int mixed, cudaStream_t st) {
    if (dial_mode == DIAL_LCE)
        return mixed ? launch_one<DIAL_LCE, true>(m, p, q, s, sc, st) : launch_one<DIAL_LCE, false>(m, p, q, s, sc, st);
    return mixed ? launch_one<DIAL_ARRAYS, true>(m, p, q, s, sc, st) : launch_one<DIAL_ARRAYS, false>(m, p, q, s, sc, st);
}

}  // namespace msb
