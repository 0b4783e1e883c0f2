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
//   aggregation group has released the group's staging area, writes its 18
//   contributions straight to their places in the chunk's sliced order (the
//   node section's dst table) and arrives on the group's stage_full barrier.
//
//   the aggregation warpgroup takes the chunks in order: it waits for a
//   chunk's staging area and adds the chunk's runs to the tile's per-node
//   accumulators in shared memory, one thread per run (a run is one node's
//   entries in ascending triangle order).  In the sliced order entry u of
//   run r sits at slice_off[r / 32] + 32 u + r % 32, so the 32 threads of a
//   warp read 32 consecutive words at every step: no bank conflicts and no
//   index loads.  When the run the plan marks as a node's last is added, the
//   node's state (position, velocity, mass, constraint flag) is copied into
//   shared memory with cp.async, and the node is finished (damping,
//   constraints, equilibrium maxima, force guard, symplectic Euler;
//   node_core) after the next chunk's runs, by which time the copy has
//   landed.  Chunks are added in order, so each node's force is the sum of
//   its contributions in ascending triangle order from zero -- the order,
//   and so the bits, of every other path.
//
// So the triangle arithmetic of the next two chunks overlaps the sums and
// node updates of the current one, and the node updates are spread over the
// tile's chunks instead of forming a phase of their own.  The scattered
// writes go to the math groups, which have time to spare; the aggregation
// group, the one that sets the pace, reads conflict-free.
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

// Aggregation warpgroups (two were measured slower on B200: 512-thread
// blocks leave the math 128 registers and it spills).
#ifndef MSB_PIPE_AGG_GROUPS
#define MSB_PIPE_AGG_GROUPS 1
#endif
constexpr int kAggThreads = 128 * MSB_PIPE_AGG_GROUPS;
constexpr int kPipeThreads = 256 + kAggThreads;
constexpr int kNsSlots = 8;   // node-section slots: a chunk's slot is refilled 8 chunks later
constexpr int kAggBar = 3;    // named barrier of the aggregation groups (1, 2: the math groups)
// Final runs per aggregation thread and chunk whose node finish is deferred.
constexpr int kDefer = MSB_PIPE_AGG_GROUPS == 1 ? 2 : 1;
constexpr int kFinWords = 8;  // prefetched node state: x, y, z, vx, vy, vz, mass, constraint word

// Shared memory: two table buffers, two sliced staging areas, the
// node-section slots, the prefetched state of deferred nodes (two chunks),
// the tile's per-node accumulators.
template <bool MIXED>
struct PipeSmem {
    using R = typename tridev::Real<MIXED>::T;
    static constexpr size_t tables = TileLayout<MIXED>::bytes;
    static constexpr size_t fin = 2 * (size_t)kDefer * kAggThreads * kFinWords * 8;
    static_assert(tables % 128 == 0 && fin % 128 == 0, "buffers stay 128-byte aligned");
    __host__ __device__ static size_t stage(int slc) { return (3 * (size_t)slc * sizeof(R) + 127) / 128 * 128; }
    __host__ __device__ static size_t ns_cap(size_t stride) { return stride - tables; }
    __host__ __device__ static size_t bytes(size_t stride, int nodes, int slc) {
        return 2 * tables + 2 * stage(slc) + kNsSlots * ns_cap(stride) + fin + 24 * (size_t)nodes;
    }
};

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
// True on every thread of a group of `count` threads (whole warps) iff `ok`
// holds on all of them.
__device__ __forceinline__ bool group_all(bool ok, int id, int count = 128) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, p;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.and.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)ok), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void group_sync(int id, int count = 128) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Asynchronous global -> shared copies of 8 and 4 bytes (this thread's own
// slots; they complete by group, in commit order).
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// All groups but the newest have landed.
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

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

// Node-section fields of a chunk (see NodeTileLayout).
struct NodeSection {
    int nruns, nent, ntri, nslices;
    const unsigned short *run_node, *run_end, *slice_off, *dst;
    __device__ __forceinline__ explicit NodeSection(const unsigned char* ns) {
        const int4 hd = *reinterpret_cast<const int4*>(ns);
        nruns = hd.x;
        nent = hd.y;
        ntri = hd.z;
        nslices = hd.w;
        run_node = reinterpret_cast<const unsigned short*>(ns + 16);
        run_end = run_node + nruns;
        slice_off = run_end + nruns + nent;
        dst = slice_off + nslices;
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
    const size_t stage_bytes = SM::stage(q.slc);
    const int slc = q.slc;  // entries per component of a sliced staging area
    unsigned char* tables = pipe_smem;
    unsigned char* stages = pipe_smem + 2 * SM::tables;
    unsigned char* nsec = stages + 2 * stage_bytes;
    double* fin = reinterpret_cast<double*>(nsec + kNsSlots * ns_cap);
    double* acc = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(fin) + SM::fin);
    const int tid = threadIdx.x, wg = tid >> 7, i = tid & 127;
    const int ia = tid - 256;  // thread of the aggregation groups
    for (int j = tid; j < 3 * q.nodes; j += kPipeThreads) acc[j] = 0.0;
    if (tid == 0) {
        for (int w = 0; w < 2; ++w) {
            mbar_init(&full[w], 1);
            mbar_init(&stage_full[w], 128);
            mbar_init(&stage_free[w], kAggThreads);
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
        R* stage = reinterpret_cast<R*>(stages + w * stage_bytes);
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
            const NodeSection ns(nsec + (size_t)(g % kNsSlots) * ns_cap);
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
            const bool live = i < ns.ntri;
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
            unsigned short dst[6];
#pragma unroll
            for (int sl = 0; sl < 6; ++sl) dst[sl] = ns.dst[sl * kTile + i];
            // The staging area is free once the aggregation group has added
            // this group's previous chunk.
            if (k > 0 && !group_all(bar_wait(&stage_free[w], (k - 1) & 1), 1 + w)) {
                if (i == 0) atomicCAS(&s.err->flag, 0, 5);
                ++k;  // the copy in flight completes phase k + 1 of `full`
                break;
            }
            // Each contribution to its node's run, in the sliced order
            // (x, y, z in three planes of slc entries); slots whose node is
            // outside the tile have none.
#pragma unroll
            for (int sl = 0; sl < 6; ++sl) {
                if (dst[sl] != 0xFFFF) {
                    stage[dst[sl]] = f[3 * sl];
                    stage[slc + dst[sl]] = f[3 * sl + 1];
                    stage[2 * slc + dst[sl]] = f[3 * sl + 2];
                }
            }
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
        // a chunk is finished one chunk later, from its state copied into
        // this thread's slot of `fin` by cp.async when its force became
        // complete.  Later final runs of a chunk (more than kDefer x 128
        // runs) are finished at once.
        const double* pos = pos_buf(s, sc.parity);
        const double* vel = vel_buf(s, sc.parity);
        const int N = m.N;
        double fmax = -1.0, vmax = -1.0;
        int fnode = INT_MAX, vnode = INT_MAX;
        int dn[kDefer];
        double dF[kDefer][3];
#pragma unroll
        for (int k = 0; k < kDefer; ++k) dn[k] = -1;
        // Run r's entries added to its node's accumulator in entry order,
        // read from the sliced staging area (consecutive words across the
        // warp); loads of four entries are issued ahead of the dependent
        // adds (same order of additions, same bits).
        auto add_run = [&](const R* stage, const NodeSection& ns, int r, int j, double& a0, double& a1,
                           double& a2) {
            const int n_e = (int)ns.run_end[r] - (r ? (int)ns.run_end[r - 1] : 0);
            const R* v = stage + ns.slice_off[r >> 5] + (r & 31);
            a0 = acc[3 * j];
            a1 = acc[3 * j + 1];
            a2 = acc[3 * j + 2];
            int u = 0;
            for (; u + 4 <= n_e; u += 4) {
                R x[4], y[4], z[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    x[k] = v[32 * (u + k)];
                    y[k] = v[slc + 32 * (u + k)];
                    z[k] = v[2 * slc + 32 * (u + k)];
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    a0 += (double)x[k];
                    a1 += (double)y[k];
                    a2 += (double)z[k];
                }
            }
            for (; u < n_e; ++u) {
                a0 += (double)v[32 * u];
                a1 += (double)v[slc + 32 * u];
                a2 += (double)v[2 * slc + 32 * u];
            }
        };
        // Node n's state into a fin slot: eight words, the last the 4-byte
        // word of the constraint flags that holds n's (the flag array is
        // padded to whole words).
        auto prefetch = [&](double* slot, int n) {
            cp_async8(slot + 0, pos + n);
            cp_async8(slot + 1, pos + N + n);
            cp_async8(slot + 2, pos + 2 * (size_t)N + n);
            cp_async8(slot + 3, vel + n);
            cp_async8(slot + 4, vel + N + n);
            cp_async8(slot + 5, vel + 2 * (size_t)N + n);
            cp_async8(slot + 6, m.mass + n);
            cp_async4(slot + 7, m.fixed + (n & ~3));
        };
        auto from_slot = [&](const double* slot, int n) {
            NodeIn in;
            in.px = slot[0];
            in.py = slot[1];
            in.pz = slot[2];
            in.vx = slot[3];
            in.vy = slot[4];
            in.vz = slot[5];
            in.mass = slot[6];
            const unsigned word = *reinterpret_cast<const unsigned*>(slot + 7);
            in.fixed = (word >> (8 * (n & 3))) & 0xffu;
            return in;
        };
        Cursor cur;
        cur.start(q);
        bool aborted = false;
        int g = 0;
        for (; cur.valid(q); ++g, cur.next(q)) {
            const int w = g & 1;
            if (!group_all(bar_wait(&stage_full[w], (g >> 1) & 1), kAggBar, kAggThreads)) {
                if (ia == 0) atomicCAS(&s.err->flag, 0, 5);
                aborted = true;
                break;
            }
            const R* stage = reinterpret_cast<const R*>(stages + w * stage_bytes);
            const NodeSection ns(nsec + (size_t)(g % kNsSlots) * ns_cap);
            const int n0 = cur.tile * q.nodes;
            double* fin_now = fin + (size_t)(g & 1) * kDefer * kAggThreads * kFinWords;
            double* fin_prev = fin + (size_t)((g & 1) ^ 1) * kDefer * kAggThreads * kFinWords;
            int cn[kDefer];
            double cF[kDefer][3];
#pragma unroll
            for (int k = 0; k < kDefer; ++k) {
                cn[k] = -1;
                const int r = ia + kAggThreads * k;
                if (r < ns.nruns) {
                    const unsigned u = ns.run_node[r];
                    const int j = u & ~kRunFinal;
                    double a0, a1, a2;
                    add_run(stage, ns, r, j, a0, a1, a2);
                    if (u & kRunFinal) {
                        // The node's force is complete: clear its
                        // accumulator for the block's next tile, start
                        // copying its state, finish it after the next chunk.
                        acc[3 * j] = acc[3 * j + 1] = acc[3 * j + 2] = 0.0;
                        cn[k] = n0 + j;
                        cF[k][0] = a0;
                        cF[k][1] = a1;
                        cF[k][2] = a2;
                        prefetch(fin_now + ((size_t)k * kAggThreads + ia) * kFinWords, n0 + j);
                    } else {
                        acc[3 * j] = a0;
                        acc[3 * j + 1] = a1;
                        acc[3 * j + 2] = a2;
                    }
                }
            }
            cp_async_commit();  // one group per chunk, empty or not
            for (int r = ia + kAggThreads * kDefer; r < ns.nruns; r += kAggThreads) {
                const unsigned u = ns.run_node[r];
                const int j = u & ~kRunFinal;
                double a0, a1, a2;
                add_run(stage, ns, r, j, a0, a1, a2);
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
            // This chunk's node-section slot and staging area are reused.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&stage_free[w]);
            // The previous chunk's deferred nodes: their state has landed.
            cp_async_wait_prev();
#pragma unroll
            for (int k = 0; k < kDefer; ++k) {
                if (dn[k] >= 0)
                    node_core(m, s, sc, gstep, dn[k], from_slot(fin_prev + ((size_t)k * kAggThreads + ia) * kFinWords, dn[k]),
                              dF[k][0], dF[k][1], dF[k][2], fmax, fnode, vmax, vnode);
                dn[k] = cn[k];
                dF[k][0] = cF[k][0];
                dF[k][1] = cF[k][1];
                dF[k][2] = cF[k][2];
            }
            // The next chunk's runs may add to the same nodes.
            group_sync(kAggBar, kAggThreads);
        }
        cp_async_wait_all();
        if (!aborted && g > 0) {
            // The last chunk's (the (g-1)-th) deferred nodes.
            const double* fin_last = fin + (size_t)((g - 1) & 1) * kDefer * kAggThreads * kFinWords;
#pragma unroll
            for (int k = 0; k < kDefer; ++k)
                if (dn[k] >= 0)
                    node_core(m, s, sc, gstep, dn[k], from_slot(fin_last + ((size_t)k * kAggThreads + ia) * kFinWords, dn[k]),
                              dF[k][0], dF[k][1], dF[k][2], fmax, fnode, vmax, vnode);
        }
        if (sc.check) {
            // Block max/argmax over the aggregation group, then the grid fold.
            constexpr int kAggWarps = kAggThreads / 32;
            __shared__ double sf[kAggWarps], sv[kAggWarps];
            __shared__ int sfn[kAggWarps], svn[kAggWarps];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double of = __shfl_down_sync(0xffffffffu, fmax, o);
                const int ofn = __shfl_down_sync(0xffffffffu, fnode, o);
                const double ov = __shfl_down_sync(0xffffffffu, vmax, o);
                const int ovn = __shfl_down_sync(0xffffffffu, vnode, o);
                eq_merge(fmax, fnode, of, ofn);
                eq_merge(vmax, vnode, ov, ovn);
            }
            const int lane = ia & 31, warp = ia >> 5;
            if (lane == 0) {
                sf[warp] = fmax;
                sfn[warp] = fnode;
                sv[warp] = vmax;
                svn[warp] = vnode;
            }
            group_sync(kAggBar, kAggThreads);
            if (ia == 0) {
                EqPartial r{sf[0], sv[0], sfn[0], svn[0]};
                for (int k = 1; k < kAggWarps; ++k) {
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
    k_node_pipe<DIAL, MIXED>
        <<<grid, kPipeThreads, PipeSmem<MIXED>::bytes(q.stride, q.nodes, q.slc), st>>>(m, p, q, s, sc);
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

size_t node_pipe_smem(size_t stride, int nodes, int slc, int mixed) {
    return mixed ? PipeSmem<true>::bytes(stride, nodes, slc) : PipeSmem<false>::bytes(stride, nodes, slc);
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
