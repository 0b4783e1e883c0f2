// C ABI of the force-and-dynamics loop (include/morphoshell_gpu.h): device
// memory ownership, the one-call-per-reference-function path, the fused
// stepper captured in CUDA graphs, and the output diagnostics.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/morphoshell_gpu.h"
#include "internal.cuh"
#include "tri_physics.cuh"

using namespace msb;

namespace {

// Steps per captured graph chunk (even, so every chunk starts on the same
// ping-pong buffer).
constexpr int kChunk = 128;

struct GraphKey {
    int len, parity, dial_mode, gd, check_last;
    double dt, damping;
    bool operator==(const GraphKey& o) const {
        return len == o.len && parity == o.parity && dial_mode == o.dial_mode && gd == o.gd &&
               check_last == o.check_last && dt == o.dt && damping == o.damping;
    }
};

struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    long long last_use;
};

}  // namespace

struct ms_handle {
    int device = 0;
    int precision = 0;
    cudaStream_t stream = nullptr;
    DevMesh m{};
    DevState s{};
    ms_params params{};
    double rho_hh = 0, force_limit = 0;
    int cur = 0;  // buffer holding the current state
    // dialling
    int protocol = 1;
    double spacing = 1.0;
    int from_ansatz = 0;
    bool programmed = false;
    // The fused protocol-3 steps dial inside the force kernel and never write
    // abar/bbar.  After them the arrays are stale: they are brought to the
    // last step's dial factor (stale_dial) by the dialling kernel only when a
    // call reads them (materialise_programmed), not after every ms_step_n.
    bool ab_stale = false;
    double stale_dial = 0.0;
    // allocations
    std::vector<void*> allocs;
    double* d_dials = nullptr;
    int dials_cap = 0;
    double* h_dials = nullptr;  // pinned
    int h_dials_cap = 0;
    DevError* h_err = nullptr;  // pinned mirror
    DevEquil* h_equil = nullptr;
    double* d_scratch_tri = nullptr;  // [2][T]
    double* d_scratch_node = nullptr; // [N]
    double* d_sum_partial = nullptr;  // [512]
    double* d_sums = nullptr;         // [4]
    double* d_out = nullptr;          // generic output staging, sized on demand
    size_t out_cap = 0;
    std::vector<GraphEntry> graphs;
    long long use_clock = 0;
    std::string last_error;
    // cluster-tiled step
    ClusterPlan plan{};
    bool have_plan = false;
    bool have_cluster = false;
    int step_path = 1;  // 0 cluster-tiled, 1 two-kernel, 2 two-kernel with bulk-copied tiles, 3 node-tiled,
                        // 4 node-tiled with warp-specialised roles
    std::vector<double> area_host;
    double lce_lam_final = 0, lce_nu = 0;
    int halo_parts = 0;
    // bulk-copy-fed per-triangle kernel
    bool have_tiles = false;
    unsigned char* d_tiles = nullptr;
    size_t tile_bytes = 0;
    // node-tiled step
    bool have_ntiles = false;
    bool have_pipe = false;  // warp-specialised node-tiled step
    NodeTilePlan ntp{};
    unsigned char* d_nt_rec = nullptr;
    std::vector<int> nt_chunk_tri;  // host copy of NodeTilePlan::chunk_tri
};

namespace {

ms_status fail(ms_handle* h, ms_status st, const std::string& msg) {
    if (h) h->last_error = msg;
    return st;
}

ms_status cuda_fail(ms_handle* h, cudaError_t e, const char* what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return fail(h, MS_ERR_OUT_OF_MEMORY, msg);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return fail(h, MS_ERR_NO_DEVICE, msg);
    return fail(h, MS_ERR_CUDA, msg);
}

#define MS_CUDA(h, call)                                     \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

template <typename T>
ms_status dalloc(ms_handle* h, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc");
    h->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return MS_OK;
}

#define MS_TRY(expr)                   \
    do {                               \
        ms_status st_ = (expr);        \
        if (st_ != MS_OK) return st_;  \
    } while (0)

void clear_graphs(ms_handle* h) {
    for (auto& g : h->graphs) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
}

// Transpose a row-major rows x cols host array into [cols][rows] on the device.
template <typename T>
ms_status upload_transposed(ms_handle* h, T* dst, const T* src, size_t rows, int cols) {
    std::vector<T> tmp(rows * cols);
    for (size_t r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) tmp[(size_t)c * rows + r] = src[r * cols + c];
    MS_CUDA(h, cudaMemcpy(dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MS_OK;
}

template <typename T>
ms_status download_transposed(ms_handle* h, T* dst, const T* src_dev, size_t rows, int cols) {
    std::vector<T> tmp(rows * cols);
    MS_CUDA(h, cudaMemcpy(tmp.data(), src_dev, tmp.size() * sizeof(T), cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) dst[r * cols + c] = tmp[(size_t)c * rows + r];
    return MS_OK;
}

ms_status reset_error(ms_handle* h) {
    DevError z{};
    z.flag = 0;
    z.base = 0;
    z.guard_key = ~0ULL;
    MS_CUDA(h, cudaMemcpyAsync(h->s.err, &z, sizeof(DevError), cudaMemcpyHostToDevice, h->stream));
    return MS_OK;
}

ms_status ensure_out(ms_handle* h, size_t bytes) {
    if (h->out_cap >= bytes) return MS_OK;
    if (h->d_out) {
        cudaFree(h->d_out);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->d_out), h->allocs.end());
        h->d_out = nullptr;
    }
    MS_TRY(dalloc(h, reinterpret_cast<char**>(&h->d_out), bytes));
    h->out_cap = bytes;
    return MS_OK;
}

bool lce_fusable(const ms_handle* h) { return h->protocol == 3 && !h->from_ansatz && h->precision >= 0; }

// Paths 3 and 4 run the whole step in one kernel.
bool one_kernel_step(const ms_handle* h) {
    return (h->step_path == 3 && h->have_ntiles) || (h->step_path == 4 && h->have_pipe);
}

// Brings abar/bbar up to the dial factor of the last fused step, as
// do_dialling (do_dialling.cpp:112-123) would have left them, before a call
// that reads them.  Enqueued on the handle's stream; no synchronisation.
ms_status materialise_programmed(ms_handle* h) {
    if (!h->ab_stale) return MS_OK;
    MS_CUDA(h, launch_dialling(h->m, h->protocol, h->stale_dial, h->spacing, h->from_ansatz, h->stream));
    h->ab_stale = false;
    return MS_OK;
}

template <typename T>
ms_status upload(ms_handle* h, T** dst, const std::vector<T>& src) {
    MS_TRY(dalloc(h, dst, src.size()));
    if (!src.empty()) MS_CUDA(h, cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MS_OK;
}

// Tile records of the bulk-copy-fed per-triangle kernel (ClusterPlan::tiles):
// ids and weights now, area in the trigonometry block (cos^2 = 1, the rest
// 0) until prepare_lce_tables writes the director's values.
ms_status build_tiles(ms_handle* h, const ms_mesh_desc* d) {
    const int T = d->num_tris;
    const int mixed = h->precision == MS_PRECISION_MIXED;
    int blocks = 0;
    if (prepare_tile_kernels(mixed, &blocks) != cudaSuccess || blocks <= 0) {
        cudaGetLastError();
        h->have_tiles = false;
        return MS_OK;  // the other paths remain
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t rec = tile_record_bytes(mixed);
    const int ntiles = (T + kTile - 1) / kTile;
    std::vector<unsigned char> buf(rec * ntiles, 0);
    const size_t ids_b = 6 * kTile * 4, coef_b = 24 * kTile * (mixed ? 4 : 8);
    for (int tile = 0; tile < ntiles; ++tile) {
        unsigned char* r = buf.data() + rec * tile;
        int32_t* ids = reinterpret_cast<int32_t*>(r);
        double* aux = reinterpret_cast<double*>(r + ids_b + coef_b);
        for (int i = 0; i < kTile; ++i) {
            const int t = tile * kTile + i;
            if (t >= T) break;
            for (int k = 0; k < 6; ++k) ids[k * kTile + i] = d->patch_ids[6LL * t + k];
            const double* w = d->deriv_coeffs + 24LL * t;
            if (mixed) {
                float* c = reinterpret_cast<float*>(r + ids_b);
                for (int k = 0; k < 24; ++k) c[k * kTile + i] = (float)w[k];
            } else {
                double* c = reinterpret_cast<double*>(r + ids_b);
                for (int k = 0; k < 24; ++k) c[k * kTile + i] = w[k];
            }
            aux[i] = d->ref_area[t];
            aux[kTile + i] = 1.0;
        }
    }
    unsigned char* dt;
    MS_TRY(upload(h, &dt, buf));
    h->d_tiles = dt;
    h->tile_bytes = rec;
    if (mixed) h->plan.tiles_f = dt;
    else h->plan.tiles = dt;
    h->plan.tile_grid = sms * blocks;
    h->have_tiles = true;
    h->step_path = 2;  // measured fastest on B200 (same bits as path 1)
    return MS_OK;
}

// Largest nodes per tile of the node-tiled step (3 FP64 or 5 mixed blocks
// per SM; the tile count is a multiple of the resident blocks).  Measured on
// the 1.8M-triangle disk: FP64 tiles of 1,023 nodes (two per block, 17.5 %
// of the triangles on borders) beat 682 (three per block) by 3.4 % and 2,046
// (one per block) by 17 %; mixed tiles of 614 nodes at 5 blocks per SM beat
// 410 at 5 and 768 at 4.  The smallest tiles worth their border: 256 nodes.
#ifndef MSB_NT_NODES
#define MSB_NT_NODES 1100
#endif
#ifndef MSB_NT_NODES_MIXED
#define MSB_NT_NODES_MIXED 1008
#endif
constexpr int kNtNodesMin = 256;
// Largest nodes per tile of the warp-specialised step (one block per SM): its
// shared memory holds two table buffers, two staging areas, eight node
// sections and the prefetched node state besides the accumulators, and tiles
// this size leave about 14 % of the triangles on tile borders.
#ifndef MSB_PIPE_NODES
#define MSB_PIPE_NODES 1600
#endif

// Plan of the node-tiled step: the chunk records, area in the trigonometry
// block (cos^2 = 1, the rest 0) until prepare_lce_tables writes the
// director's values.  A block walks its tiles in turn, so the step takes as
// long as the block with the most tiles: the tile size is chosen so that the
// tile count is a multiple of the resident blocks (SMs x blocks per SM), at
// the largest size that keeps those blocks resident.  Leaves the other paths
// in place when the kernel cannot be set up.
ms_status build_node_tiles(ms_handle* h, const ms_mesh_desc* d, const std::vector<int>& off,
                           const std::vector<int>& ent) {
    const int mixed = h->precision == MS_PRECISION_MIXED;
    const int N = d->num_nodes, T = d->num_tris;
    if (N <= 0 || T <= 0) return MS_OK;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    NodeTileLayout L;
    std::string err;
    int NT = 0, blocks = 0, pipe_blocks = 0;
    auto tile_smem = [&](const NodeTileLayout& lay, int nodes) { return node_tile_smem(lay.stride, nodes, mixed); };
    auto pipe_smem = [&](const NodeTileLayout& lay, int nodes) {
        return node_pipe_smem(lay.stride, nodes, lay.slc_max, mixed);
    };
    auto tile_blocks = [&](size_t smem) {
        int b = 0;
        if (prepare_node_tile_kernels(mixed, smem, &b) != cudaSuccess) {
            cudaGetLastError();
            b = 0;
        }
        return b;
    };
    auto pipe_blocks_for = [&](size_t smem) {
        int b = 0;
        if (prepare_node_pipe_kernels(mixed, smem, &b) != cudaSuccess) {
            cudaGetLastError();
            b = 0;
        }
        return b;
    };
    // One plan serves both node-tiled kernels.  By default its tiles are
    // sized for the node-tiled kernel (path 3, the faster on B200) and its
    // records carry no sliced order, so path 4 is not offered.  With
    // MSB_NODE_TILE_PLAN=4 in the environment the tiles are sized for the
    // warp-specialised kernel (path 4, one block per SM) and the records
    // carry the sliced order it reads; path 3 runs on that plan too.
    const char* plan_env = std::getenv("MSB_NODE_TILE_PLAN");
    const bool plan4 = plan_env && std::string(plan_env) == "4";
    if (plan4) {
        if (!choose_node_tiles(d->patch_ids, N, T, mixed, sms, 1, MSB_PIPE_NODES, kNtNodesMin, off, ent, pipe_smem,
                               pipe_blocks_for, L, NT, pipe_blocks, err, 1))
            return fail(h, MS_ERR_INVALID_ARGUMENT, err);
        if (pipe_blocks > 0) blocks = tile_blocks(tile_smem(L, NT));
    }
    if (pipe_blocks <= 0) {
        // MSB_NT_NODES in the environment overrides the largest tile (a
        // tuning knob; the plan still picks a tile count that is a multiple
        // of the resident blocks).
        int nt_max = mixed ? MSB_NT_NODES_MIXED : MSB_NT_NODES;
        if (const char* e = std::getenv("MSB_NT_NODES")) nt_max = std::max(kNtNodesMin, std::atoi(e));
        if (!choose_node_tiles(d->patch_ids, N, T, mixed, sms, node_tile_blocks_target(mixed), nt_max, kNtNodesMin,
                               off, ent, tile_smem, tile_blocks, L, NT, blocks, err, 0))
            return fail(h, MS_ERR_INVALID_ARGUMENT, err);
    }
    if (blocks <= 0 && pipe_blocks <= 0) {
        h->have_ntiles = false;
        return MS_OK;  // the other paths remain
    }
    const int K = L.K, C = L.C;
    const size_t stride = L.stride;
    std::vector<unsigned char> buf;
    std::vector<int>& ctri = h->nt_chunk_tri;
    fill_node_tile_records(L, d->patch_ids, d->deriv_coeffs, nullptr, d->ref_area, nullptr, mixed, buf, ctri);
    unsigned char* d_rec;
    int *d_tile_chunk, *d_ctri;
    unsigned* d_bytes;
    MS_TRY(upload(h, &d_rec, buf));
    MS_TRY(upload(h, &d_tile_chunk, L.tile_chunk));
    MS_TRY(upload(h, &d_bytes, L.bytes));
    MS_TRY(upload(h, &d_ctri, ctri));
    NodeTilePlan& q = h->ntp;
    q.nodes = NT;
    q.ntiles = K;
    q.nchunks = C;
    q.grid = sms * blocks;
    q.grid_pipe = sms * std::min(pipe_blocks, 1);
    q.stride = stride;
    q.slc = L.slc_max;
    q.rec = d_rec;
    q.tile_chunk = d_tile_chunk;
    q.chunk_bytes = d_bytes;
    q.chunk_tri = d_ctri;
    q.chunk_tag = nullptr;
    h->d_nt_rec = d_rec;
    // One equilibrium partial per block.
    const int parts = std::min(K, std::max(q.grid, q.grid_pipe));
    if (parts > h->s.eq_blocks) {
        EqPartial* ep;
        MS_TRY(dalloc(h, &ep, parts));
        h->s.eq_part = ep;
        h->s.eq_blocks = parts;
    }
    h->have_ntiles = q.grid > 0;
    h->have_pipe = q.grid_pipe > 0;
    // The node-tiled kernels once every block has a tile of its own (same
    // bits as paths 1 and 2); the warp-specialised one when its plan was
    // asked for.
    if (h->have_pipe && K >= q.grid_pipe) h->step_path = 4;
    else if (h->have_ntiles && K >= q.grid) h->step_path = 3;
    return MS_OK;
}

// Tiles of cs * tpc consecutive triangles, one per thread-block cluster; a
// node is owned by a tile when all its incidences lie in it (see
// ClusterPlan).  Falls back to the two-kernel step when cluster launches are
// unavailable.
ms_status build_cluster_plan(ms_handle* h, const ms_mesh_desc* d, const std::vector<int>& off,
                             const std::vector<int>& ent) {
    const int N = d->num_nodes, T = d->num_tris;
    const int tpc = 768;
    // The per-triangle tables below serve both paths; the tiling only the
    // cluster path, which needs cluster launches.
    h->have_cluster = prepare_cluster_kernels(tpc) == cudaSuccess;
    cudaGetLastError();
    const int cs = h->have_cluster ? choose_cluster_size(tpc, cluster_threads(), h->precision) : 1;
    ClusterPlan& p = h->plan;
    p.cs = cs;
    p.tpc = tpc;
    p.threads = cluster_threads();
    const int ct = cs * tpc;
    p.nclusters = (T + ct - 1) / ct;
    std::vector<int> owner(N, -1);
    for (int n = 0; n < N; ++n) {
        if (off[n] == off[n + 1]) continue;
        const int c0 = (ent[off[n]] / 6) / ct, c1 = (ent[off[n + 1] - 1] / 6) / ct;
        if (c0 == c1) owner[n] = c0;
    }
    std::vector<int> own_base(p.nclusters + 1, 0), own_nodes, own_off, halo_nodes;
    std::vector<unsigned short> own_ent;
    for (int n = 0; n < N; ++n)
        if (owner[n] >= 0) own_base[owner[n] + 1] += 1;
    for (int c = 0; c < p.nclusters; ++c) own_base[c + 1] += own_base[c];
    own_nodes.assign(own_base[p.nclusters], 0);
    {
        std::vector<int> fill(own_base.begin(), own_base.end() - 1);
        for (int n = 0; n < N; ++n)
            if (owner[n] >= 0) own_nodes[fill[owner[n]]++] = n;
            else halo_nodes.push_back(n);
    }
    own_off.reserve(own_nodes.size() + 1);
    own_off.push_back(0);
    std::vector<int32_t> idx(8ULL * T, 0);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 6; ++k) idx[8ULL * t + k] = d->patch_ids[6ULL * t + k];
    for (size_t i = 0; i < own_nodes.size(); ++i) {
        const int n = own_nodes[i], c = owner[n];
        for (int k = off[n]; k < off[n + 1]; ++k) {
            const int t = ent[k] / 6, slot = ent[k] % 6;
            const int lt = t - c * ct, rank = lt / tpc, li = lt % tpc;
            own_ent.push_back((unsigned short)((rank << 13) | (li << 3) | slot));
        }
        own_off.push_back((int)own_ent.size());
    }
    for (int n : halo_nodes)
        for (int k = off[n]; k < off[n + 1]; ++k) idx[8ULL * (ent[k] / 6) + 6] |= 1 << (ent[k] % 6);
    int4* tri_idx;
    double* coef_aos;
    int *d_own_base, *d_own_nodes, *d_own_off, *d_halo;
    unsigned short* d_own_ent;
    MS_TRY(dalloc(h, &tri_idx, 2ULL * T));
    MS_CUDA(h, cudaMemcpy(tri_idx, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    MS_TRY(dalloc(h, &coef_aos, 24ULL * T));
    MS_CUDA(h, cudaMemcpy(coef_aos, d->deriv_coeffs, 24ULL * T * sizeof(double), cudaMemcpyHostToDevice));
    if (h->precision == MS_PRECISION_MIXED) {
        std::vector<float> cf(24ULL * T);
        for (size_t k = 0; k < cf.size(); ++k) cf[k] = (float)d->deriv_coeffs[k];
        float* coef_f;
        MS_TRY(upload(h, &coef_f, cf));
        p.coef_aos_f = coef_f;
    }
    MS_TRY(upload(h, &d_own_base, own_base));
    MS_TRY(upload(h, &d_own_nodes, own_nodes));
    MS_TRY(upload(h, &d_own_off, own_off));
    MS_TRY(upload(h, &d_own_ent, own_ent));
    MS_TRY(upload(h, &d_halo, halo_nodes));
    p.tri_idx = tri_idx;
    p.coef_aos = coef_aos;
    p.own_base = d_own_base;
    p.own_nodes = d_own_nodes;
    p.own_off = d_own_off;
    p.own_ent = d_own_ent;
    p.halo_nodes = d_halo;
    p.n_halo = (int)halo_nodes.size();
    // Equilibrium partials: one per cluster-kernel CTA plus one per halo block.
    h->halo_parts = p.n_halo > 0 ? (p.n_halo + 255) / 256 : 1;
    const int parts = p.nclusters * p.cs + h->halo_parts;
    if (parts > h->s.eq_blocks) {
        EqPartial* ep;
        MS_TRY(dalloc(h, &ep, parts));
        h->s.eq_part = ep;
        h->s.eq_blocks = parts;
    }
    h->have_plan = true;
    MS_TRY(build_tiles(h, d));
    return build_node_tiles(h, d, off, ent);
}

// Per-triangle director trigonometry for the cluster kernel's protocol-3
// dialling, and whether lambda_final and nu_ot are uniform (then lambda and
// lambda^(-2 nu) are per-step scalars computed on the host).
ms_status prepare_lce_tables(ms_handle* h, const double* info, int ka) {
    if (!h->have_plan || h->protocol != 3 || ka < 3) return MS_OK;
    const int T = h->m.T;
    std::vector<double> aux(4ULL * T), ln(2ULL * T);
    bool uniform = true;
    for (int t = 0; t < T; ++t) {
        const double ang = info[(size_t)t * ka], c = std::cos(ang), s = std::sin(ang);
        aux[4ULL * t] = h->area_host[t];
        aux[4ULL * t + 1] = c * c;
        aux[4ULL * t + 2] = s * s;
        aux[4ULL * t + 3] = c * s;
        ln[2ULL * t] = info[(size_t)t * ka + 1];
        ln[2ULL * t + 1] = info[(size_t)t * ka + 2];
        uniform = uniform && ln[2ULL * t] == ln[0] && ln[2ULL * t + 1] == ln[1];
    }
    double4* d_aux;
    double2* d_ln;
    MS_TRY(dalloc(h, &d_aux, T));
    MS_CUDA(h, cudaMemcpy(d_aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice));
    MS_TRY(dalloc(h, &d_ln, T));
    MS_CUDA(h, cudaMemcpy(d_ln, ln.data(), ln.size() * sizeof(double), cudaMemcpyHostToDevice));
    h->plan.tri_aux = d_aux;
    h->plan.lce_ln = d_ln;
    if (h->have_tiles) {
        // The trigonometry block of every tile record: [4][kTile] doubles.
        const int ntiles = (T + kTile - 1) / kTile;
        std::vector<double> blk(4ULL * kTile * ntiles, 0.0);
        for (int t = 0; t < T; ++t) {
            const int tile = t / kTile, i = t % kTile;
            for (int k = 0; k < 4; ++k) blk[(size_t)tile * 4 * kTile + k * kTile + i] = aux[4ULL * t + k];
        }
        const size_t off = 6 * kTile * 4 + 24 * kTile * (h->precision == MS_PRECISION_MIXED ? 4 : 8);
        MS_CUDA(h, cudaMemcpy2D(h->d_tiles + off, h->tile_bytes, blk.data(), 4 * kTile * sizeof(double),
                                4 * kTile * sizeof(double), ntiles, cudaMemcpyHostToDevice));
    }
    if (h->have_ntiles) {
        const int C = h->ntp.nchunks;
        std::vector<double> blk(4ULL * kTile * C, 0.0);
        for (size_t j = 0; j < h->nt_chunk_tri.size(); ++j) {
            const int t = h->nt_chunk_tri[j];
            if (t < 0) continue;
            const size_t c = j / kTile, i = j % kTile;
            for (int k = 0; k < 4; ++k) blk[c * 4 * kTile + k * kTile + i] = aux[4ULL * t + k];
        }
        const size_t off = 6 * kTile * 4 + 24 * kTile * (h->precision == MS_PRECISION_MIXED ? 4 : 8);
        MS_CUDA(h, cudaMemcpy2D(h->d_nt_rec + off, h->ntp.stride, blk.data(), 4 * kTile * sizeof(double),
                                4 * kTile * sizeof(double), C, cudaMemcpyHostToDevice));
    }
    h->plan.lce_uniform = uniform ? 1 : 0;
    h->lce_lam_final = ln[0];
    h->lce_nu = ln[1];
    return MS_OK;
}

bool use_cluster(const ms_handle* h, bool dialling) {
    if (!h->have_plan || !h->have_cluster || h->step_path != 0) return false;
    if (dialling && !lce_fusable(h)) return false;
    if (dialling && !h->plan.tri_aux) return false;
    return true;
}

}  // namespace

extern "C" {

const char* ms_status_string(int st) {
    switch (st) {
        case MS_OK: return "ok";
        case MS_ERR_INVALID_ARGUMENT: return "invalid argument";
        case MS_ERR_CUDA: return "CUDA error";
        case MS_ERR_IMPLAUSIBLE_FORCE: return "implausibly_high_force";
        case MS_ERR_NON_FINITE: return "non-finite value";
        case MS_ERR_TIMEOUT: return "timeout";
        case MS_ERR_NO_DEVICE: return "no CUDA device";
        case MS_ERR_OUT_OF_MEMORY: return "out of device memory";
        case MS_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* ms_last_error(const ms_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

ms_status ms_device_info(char* buf, size_t len) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        if (buf && len) std::snprintf(buf, len, "no device: %s", cudaGetErrorString(e));
        return MS_ERR_NO_DEVICE;
    }
    cudaDeviceProp p{};
    cudaGetDeviceProperties(&p, dev);
    if (buf && len)
        std::snprintf(buf, len, "%s sm_%d%d, %d SMs, %.1f GB", p.name, p.major, p.minor, p.multiProcessorCount,
                      p.totalGlobalMem / 1e9);
    return MS_OK;
}

ms_status ms_create(const ms_mesh_desc* d, const ms_params* prm, int device, int precision, ms_handle** out) {
    if (!out) return MS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!d || !prm || d->num_nodes <= 0 || d->num_tris <= 0 || !d->patch_ids || !d->deriv_coeffs || !d->ref_area ||
        !d->ref_thickness || !d->ref_shear_modulus || !d->node_mass || !d->is_constrained)
        return MS_ERR_INVALID_ARGUMENT;
    if (precision != MS_PRECISION_FP64 && precision != MS_PRECISION_MIXED) return MS_ERR_INVALID_ARGUMENT;
    const int N = d->num_nodes, T = d->num_tris;
    for (long long k = 0; k < 6LL * T; ++k)
        if (d->patch_ids[k] < 0 || d->patch_ids[k] >= N) return MS_ERR_INVALID_ARGUMENT;
    if ((long long)6 * T >= (1LL << 31)) return MS_ERR_UNSUPPORTED;

    ms_handle* h = new ms_handle();
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        delete h;
        return MS_ERR_NO_DEVICE;
    }
    if (device >= 0) {
        if (device >= ndev) {
            delete h;
            return MS_ERR_INVALID_ARGUMENT;
        }
        cudaSetDevice(device);
    }
    cudaGetDevice(&h->device);
    h->precision = precision;
    h->params = *prm;
    h->rho_hh = prm->ref_density * prm->min_ref_thickness * prm->min_ref_thickness;
    h->force_limit = 50000.0 * prm->char_force_scale;
    auto bail = [&](ms_status st) {
        ms_destroy(h);
        return st;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MS_ERR_CUDA);

    DevMesh& m = h->m;
    DevState& s = h->s;
    m.N = N;
    m.T = T;
    m.nu = prm->def_poisson_ratio;
    m.gamma = prm->bend_stiffening_scale_factor;
    int* patch;
    double *coef, *area, *thick, *shear, *mass;
    unsigned char *fixed, *boundary = nullptr;
    ms_status st;
    if ((st = dalloc(h, &patch, 6ULL * T)) || (st = dalloc(h, &coef, 24ULL * T)) || (st = dalloc(h, &area, T)) ||
        (st = dalloc(h, &thick, T)) || (st = dalloc(h, &shear, T)) || (st = dalloc(h, &mass, N)) ||
        (st = dalloc(h, &fixed, N + 4)))
        return bail(st);
    if ((st = upload_transposed<int>(h, patch, d->patch_ids, T, 6)) ||
        (st = upload_transposed<double>(h, coef, d->deriv_coeffs, T, 24)))
        return bail(st);
    if (cudaMemcpy(area, d->ref_area, sizeof(double) * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(thick, d->ref_thickness, sizeof(double) * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(shear, d->ref_shear_modulus, sizeof(double) * T, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(mass, d->node_mass, sizeof(double) * N, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(fixed, d->is_constrained, N, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(fixed + N, 0, 4) != cudaSuccess)  // whole 4-byte words are read around the last nodes
        return bail(MS_ERR_CUDA);
    if (d->is_boundary) {
        if ((st = dalloc(h, &boundary, N))) return bail(st);
        if (cudaMemcpy(boundary, d->is_boundary, N, cudaMemcpyHostToDevice) != cudaSuccess) return bail(MS_ERR_CUDA);
    }
    m.patch = patch;
    m.coef = coef;
    m.area = area;
    m.thick = thick;
    m.shear = shear;
    m.mass = mass;
    m.fixed = fixed;
    m.boundary = boundary;
    bool uniform = true;
    for (int t = 1; t < T && uniform; ++t)
        uniform = d->ref_thickness[t] == d->ref_thickness[0] && d->ref_shear_modulus[t] == d->ref_shear_modulus[0];
    m.uniform_hmu = uniform ? 1 : 0;
    m.h_uniform = d->ref_thickness[0];
    m.mu_uniform = d->ref_shear_modulus[0];
    dev::material_coefs(m.h_uniform, m.mu_uniform, m.nu, m.gamma, m.ks_uniform, m.kb_uniform, m.igmh_uniform);

    // Incidence lists: node -> (6t + slot), ascending t.
    std::vector<int> off(N + 1, 0), ent(6ULL * T);
    {
        for (long long k = 0; k < 6LL * T; ++k) off[d->patch_ids[k] + 1] += 1;
        for (int n = 0; n < N; ++n) off[n + 1] += off[n];
        std::vector<int> fill(off.begin(), off.end() - 1);
        for (int t = 0; t < T; ++t)
            for (int k = 0; k < 6; ++k) ent[fill[d->patch_ids[6 * t + k]]++] = 6 * t + k;
        int *doff, *dent;
        if ((st = dalloc(h, &doff, N + 1)) || (st = dalloc(h, &dent, 6ULL * T))) return bail(st);
        if (cudaMemcpy(doff, off.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dent, ent.data(), sizeof(int) * 6 * (size_t)T, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(MS_ERR_CUDA);
        m.inc_off = doff;
        m.inc_ent = dent;
        std::vector<int> soff, sent;
        build_sell(N, off.data(), ent.data(), soff, sent);
        int *dsoff, *dsent;
        if ((st = upload(h, &dsoff, soff)) || (st = upload(h, &dsent, sent))) return bail(st);
        m.sell_off = dsoff;
        m.sell_ent = dsent;
    }
    // Programmed tensors: flat reference state until ms_set_programmed.
    double *abar, *bbar, *a0, *b0;
    if ((st = dalloc(h, &abar, 3ULL * T)) || (st = dalloc(h, &bbar, 3ULL * T)) || (st = dalloc(h, &a0, 3ULL * T)) ||
        (st = dalloc(h, &b0, 3ULL * T)))
        return bail(st);
    {
        std::vector<double> ident(3ULL * T, 0.0);
        for (int t = 0; t < T; ++t) {
            ident[t] = 1.0;
            ident[2ULL * T + t] = 1.0;
        }
        cudaMemcpy(abar, ident.data(), sizeof(double) * 3 * T, cudaMemcpyHostToDevice);
        cudaMemcpy(a0, ident.data(), sizeof(double) * 3 * T, cudaMemcpyHostToDevice);
        cudaMemset(bbar, 0, sizeof(double) * 3 * T);
        cudaMemset(b0, 0, sizeof(double) * 3 * T);
    }
    m.abar = abar;
    m.bbar = bbar;
    m.a0 = a0;
    m.b0 = b0;

    // State and work buffers.
    for (int b = 0; b < 2; ++b) {
        if ((st = dalloc(h, &s.pos[b], 3ULL * N)) || (st = dalloc(h, &s.vel[b], 3ULL * N))) return bail(st);
        cudaMemset(s.pos[b], 0, sizeof(double) * 3 * N);
        cudaMemset(s.vel[b], 0, sizeof(double) * 3 * N);
    }
    if ((st = dalloc(h, &s.forces, 3ULL * N)) || (st = dalloc(h, &s.cq, 15ULL * T)) ||
        (st = dalloc(h, &s.dEdcq, 15ULL * T)) || (st = dalloc(h, &s.contrib, 18ULL * T)) ||
        (st = dalloc(h, &s.err, 1)) || (st = dalloc(h, &s.equil, 1)))
        return bail(st);
    cudaMemset(s.forces, 0, sizeof(double) * 3 * N);
    s.eq_blocks = (N + 255) / 256;
    if ((st = dalloc(h, &s.eq_part, s.eq_blocks)) || (st = dalloc(h, &s.eq_counter, 1))) return bail(st);
    cudaMemset(s.eq_counter, 0, sizeof(unsigned int));
    if ((st = dalloc(h, &h->d_scratch_tri, 2ULL * T)) || (st = dalloc(h, &h->d_scratch_node, N)) ||
        (st = dalloc(h, &h->d_sum_partial, 1024)) || (st = dalloc(h, &h->d_sums, 4)))
        return bail(st);
    if (precision == MS_PRECISION_MIXED) {
        float* contrib_f;
        if ((st = dalloc(h, &contrib_f, 6ULL * kMixedSlot * T))) return bail(st);
        m.contrib_f = contrib_f;
    }
    h->area_host.assign(d->ref_area, d->ref_area + T);
    if ((st = build_cluster_plan(h, d, off, ent))) return bail(st);
    if (cudaMallocHost(&h->h_err, sizeof(DevError)) != cudaSuccess ||
        cudaMallocHost(&h->h_equil, sizeof(DevEquil)) != cudaSuccess)
        return bail(MS_ERR_CUDA);
    if (reset_error(h) != MS_OK) return bail(MS_ERR_CUDA);
    cudaError_t le = cudaStreamSynchronize(h->stream);
    if (le != cudaSuccess) {
        cuda_fail(h, le, "ms_create");
        return bail(MS_ERR_CUDA);
    }
    *out = h;
    return MS_OK;
}

ms_status ms_destroy(ms_handle* h) {
    if (!h) return MS_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    clear_graphs(h);
    for (void* p : h->allocs) cudaFree(p);
    if (h->h_dials) cudaFreeHost(h->h_dials);
    if (h->h_err) cudaFreeHost(h->h_err);
    if (h->h_equil) cudaFreeHost(h->h_equil);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MS_OK;
}

ms_status ms_upload_dofs(ms_handle* h, const double* dofs, const double* vel) {
    if (!h || !dofs) return MS_ERR_INVALID_ARGUMENT;
    const size_t n3 = 3ULL * h->m.N;
    MS_CUDA(h, cudaMemcpyAsync(h->s.pos[h->cur], dofs, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (vel) MS_CUDA(h, cudaMemcpyAsync(h->s.vel[h->cur], vel, n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    else MS_CUDA(h, cudaMemsetAsync(h->s.vel[h->cur], 0, n3 * sizeof(double), h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_download_dofs(ms_handle* h, double* dofs, double* vel) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    const size_t n3 = 3ULL * h->m.N;
    if (dofs) MS_CUDA(h, cudaMemcpyAsync(dofs, h->s.pos[h->cur], n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (vel) MS_CUDA(h, cudaMemcpyAsync(vel, h->s.vel[h->cur], n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_download_forces(ms_handle* h, double* forces) {
    if (!h || !forces) return MS_ERR_INVALID_ARGUMENT;
    MS_CUDA(h, cudaMemcpyAsync(forces, h->s.forces, 3ULL * h->m.N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_set_programmed(ms_handle* h, int protocol, const double* abar_info, int ka, const double* bbar_info,
                            int kb, double spacing, int from_ansatz) {
    if (!h || !abar_info || !bbar_info || ka <= 0 || kb <= 0) return MS_ERR_INVALID_ARGUMENT;
    const int need_a[6] = {0, 3, 3, 3, 13, 1};
    const int need_b[6] = {0, 3, 3, 1, 1, 1};
    if (protocol < 1 || protocol > 5) return fail(h, MS_ERR_INVALID_ARGUMENT, "protocol must be 1..5");
    if (ka < need_a[protocol] || kb < need_b[protocol])
        return fail(h, MS_ERR_INVALID_ARGUMENT, "abar_info/bbar_info have too few columns for this protocol");
    if (protocol == 4 && !(spacing > 0)) return fail(h, MS_ERR_INVALID_ARGUMENT, "protocol 4 needs spacing > 0");
    MS_TRY(materialise_programmed(h));
    const size_t T = h->m.T;
    if (h->m.info_a) {
        cudaFree((void*)h->m.info_a);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->m.info_a), h->allocs.end());
    }
    if (h->m.info_b) {
        cudaFree((void*)h->m.info_b);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->m.info_b), h->allocs.end());
    }
    double *ia, *ib;
    MS_TRY(dalloc(h, &ia, T * ka));
    MS_TRY(dalloc(h, &ib, T * kb));
    MS_TRY(upload_transposed<double>(h, ia, abar_info, T, ka));
    MS_TRY(upload_transposed<double>(h, ib, bbar_info, T, kb));
    h->m.info_a = ia;
    h->m.info_b = ib;
    h->m.ka = ka;
    h->m.kb = kb;
    h->protocol = protocol;
    h->spacing = spacing;
    h->from_ansatz = from_ansatz ? 1 : 0;
    h->programmed = true;
    clear_graphs(h);  // graphs bake the mesh struct
    MS_TRY(prepare_lce_tables(h, abar_info, ka));
    return MS_OK;
}

ms_status ms_set_zero_dial_state(ms_handle* h, const double* a0, const double* b0) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    MS_TRY(materialise_programmed(h));
    const size_t T = h->m.T;
    std::vector<double> ident(3 * T, 0.0);
    for (size_t t = 0; t < T; ++t) {
        ident[t] = 1.0;
        ident[2 * T + t] = 1.0;
    }
    if (a0) MS_TRY(upload_transposed<double>(h, (double*)h->m.a0, a0, T, 3));
    else MS_CUDA(h, cudaMemcpy((void*)h->m.a0, ident.data(), 3 * T * sizeof(double), cudaMemcpyHostToDevice));
    if (b0) MS_TRY(upload_transposed<double>(h, (double*)h->m.b0, b0, T, 3));
    else MS_CUDA(h, cudaMemset((void*)h->m.b0, 0, 3 * T * sizeof(double)));
    return MS_OK;
}

ms_status ms_do_dialling(ms_handle* h, double dial) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    if (!h->programmed) return fail(h, MS_ERR_INVALID_ARGUMENT, "ms_set_programmed has not been called");
    MS_CUDA(h, launch_dialling(h->m, h->protocol, dial, h->spacing, h->from_ansatz, h->stream));
    h->ab_stale = false;
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_download_programmed(ms_handle* h, double* abar, double* bbar) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    MS_TRY(materialise_programmed(h));
    if (abar) MS_TRY(download_transposed<double>(h, abar, h->m.abar, h->m.T, 3));
    if (bbar) MS_TRY(download_transposed<double>(h, bbar, h->m.bbar, h->m.T, 3));
    return MS_OK;
}

ms_status ms_surface_derivs(ms_handle* h, double* cq) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    MS_CUDA(h, launch_surface_derivs(h->m, h->s, h->cur, h->stream));
    if (cq)
        MS_CUDA(h, cudaMemcpyAsync(cq, h->s.cq, 15ULL * h->m.T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_a_b_normals(ms_handle* h, double* a, double* b, double* n) {
    if (!h || !a || !b || !n) return MS_ERR_INVALID_ARGUMENT;
    const size_t T = h->m.T;
    MS_TRY(ensure_out(h, 9 * T * sizeof(double)));
    double* da = h->d_out;
    MS_CUDA(h, launch_a_b_normals(h->m, h->s, da, da + 3 * T, da + 6 * T, h->stream));
    MS_CUDA(h, cudaMemcpyAsync(a, da, 3 * T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaMemcpyAsync(b, da + 3 * T, 3 * T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaMemcpyAsync(n, da + 6 * T, 3 * T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_deformation_forces(ms_handle* h, double* forces, double* dE) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    MS_TRY(materialise_programmed(h));
    MS_CUDA(h, launch_forces_from_cq(h->m, h->s, dE ? 1 : 0, h->stream));
    MS_CUDA(h, launch_gather_forces(h->m, h->s, h->stream));
    if (forces)
        MS_CUDA(h, cudaMemcpyAsync(forces, h->s.forces, 3ULL * h->m.N * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->stream));
    if (dE)
        MS_CUDA(h, cudaMemcpyAsync(dE, h->s.dEdcq, 15ULL * h->m.T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_non_deformation_forces(ms_handle* h, double damping, int gd) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    if (!gd) MS_CUDA(h, launch_damping(h->m, h->s, h->cur, damping, h->rho_hh, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

ms_status ms_impose_constraints(ms_handle* h) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    MS_CUDA(h, launch_constraints(h->m, h->s, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

static void fill_equil(const ms_handle* h, const DevEquil& e, ms_equil_result* out) {
    out->max_force = e.max_force;
    out->max_speed = e.max_speed;
    out->max_force_node = e.max_force_node;
    out->max_speed_node = e.max_speed_node;
    out->at_equilibrium = (e.max_force / h->params.char_force_scale) < h->params.force_to_char_force_ratio_equil_threshold &&
                          (e.max_speed / h->params.char_speed_scale) < h->params.speed_to_char_speed_ratio_equil_threshold;
}

ms_status ms_is_at_equilibrium(ms_handle* h, ms_equil_result* out) {
    if (!h || !out) return MS_ERR_INVALID_ARGUMENT;
    MS_CUDA(h, launch_equilibrium(h->m, h->s, h->cur, h->stream));
    MS_CUDA(h, cudaMemcpyAsync(h->h_equil, h->s.equil, sizeof(DevEquil), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    fill_equil(h, *h->h_equil, out);
    return MS_OK;
}

ms_status ms_advance_dynamics(ms_handle* h, double dt, double damping, int gd, int64_t* bad_dof, double* bad_force) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    if (bad_dof) *bad_dof = -1;
    MS_TRY(reset_error(h));
    MS_CUDA(h, launch_guard(h->m, h->s, h->force_limit, h->stream));
    MS_CUDA(h, cudaMemcpyAsync(h->h_err, h->s.err, sizeof(DevError), cudaMemcpyDeviceToHost, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->h_err->flag) {
        const long long d = (long long)(h->h_err->guard_key & 0xffffffffULL);
        double f = 0;
        cudaMemcpy(&f, h->s.forces + d, sizeof(double), cudaMemcpyDeviceToHost);
        if (bad_dof) *bad_dof = d;
        if (bad_force) *bad_force = f;
        return fail(h, MS_ERR_IMPLAUSIBLE_FORCE, "implausibly_high_force");
    }
    MS_CUDA(h, launch_advance(h->m, h->s, h->cur, dt, damping, h->rho_hh, gd, h->stream));
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    return MS_OK;
}

// Per-step {dial, lambda, lambda^(-2 nu)} triples for the device (the last two
// are used when lambda_final and nu_ot are uniform; formed as do_dialling.cpp:116-118
// forms them, in double on the host).
static ms_status stage_dials(ms_handle* h, const double* dials, int n) {
    if (h->dials_cap < 3 * n) {
        if (h->d_dials) {
            cudaFree(h->d_dials);
            h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->d_dials), h->allocs.end());
        }
        const int cap = std::max(3 * n, 3072);
        MS_TRY(dalloc(h, &h->d_dials, cap));
        h->dials_cap = cap;
        h->s.dials = h->d_dials;
        clear_graphs(h);
    }
    if (h->h_dials_cap < 3 * n) {
        if (h->h_dials) cudaFreeHost(h->h_dials);
        const int cap = std::max(3 * n, 3072);
        MS_CUDA(h, cudaMallocHost(&h->h_dials, cap * sizeof(double)));
        h->h_dials_cap = cap;
    }
    MS_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < n; ++i) {
        const double dial = dials[i];
        const double lam = (1.0 - dial) * 1.0 + dial * h->lce_lam_final;
        h->h_dials[3 * i] = dial;
        h->h_dials[3 * i + 1] = lam;
        h->h_dials[3 * i + 2] = std::pow(lam, -2.0 * h->lce_nu);
    }
    MS_CUDA(h, cudaMemcpyAsync(h->d_dials, h->h_dials, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    return MS_OK;
}

static cudaError_t launch_step(ms_handle* h, const StepScalars& sc, bool cluster, int dial_mode, cudaStream_t st);

// The graph of one chunk of fused steps (key.len steps from buffer
// key.parity), captured on the handle's stream and cached; the cache keeps
// the eight most recently used.
static ms_status capture_steps(ms_handle* h, const GraphKey& key, bool cluster, cudaGraphExec_t* out) {
    cudaStream_t st = h->stream;
    cudaGraph_t graph;
    MS_CUDA(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    const int dial_mode = key.dial_mode & 15;
    for (int i = 0; i < key.len && ce == cudaSuccess; ++i) {
        StepScalars sc{i, key.parity ^ (i & 1), key.dt, key.damping, h->rho_hh, h->force_limit, key.gd,
                       (key.check_last && i == key.len - 1) ? 1 : 0};
        ce = launch_step(h, sc, cluster, dial_mode, st);
    }
    if (ce == cudaSuccess) ce = launch_chunk_end(h->s, key.len, st);
    cudaError_t ee = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) return cuda_fail(h, ce, "capture");
    if (ee != cudaSuccess) return cuda_fail(h, ee, "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    ee = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ee != cudaSuccess) return cuda_fail(h, ee, "cudaGraphInstantiate");
    if (h->graphs.size() >= 8) {
        auto it = std::min_element(h->graphs.begin(), h->graphs.end(),
                                   [](const GraphEntry& a, const GraphEntry& b) { return a.last_use < b.last_use; });
        cudaGraphExecDestroy(it->exec);
        h->graphs.erase(it);
    }
    h->graphs.push_back({key, exec, ++h->use_clock});
    *out = exec;
    return MS_OK;
}

// The two kernels of one fused step on the selected path.
static cudaError_t launch_step(ms_handle* h, const StepScalars& sc, bool cluster, int dial_mode, cudaStream_t st) {
    cudaError_t e;
    if (cluster) {
        e = launch_cluster_step(h->m, h->plan, h->s, sc, dial_mode, h->precision, st);
        if (e == cudaSuccess) e = launch_halo_update(h->m, h->plan, h->s, sc, h->precision, st);
    } else if (h->step_path == 4 && h->have_pipe) {
        e = launch_node_pipe(h->m, h->plan, h->ntp, h->s, sc, dial_mode, h->precision, st);
    } else if (h->step_path == 3 && h->have_ntiles) {
        e = launch_node_tiles(h->m, h->plan, h->ntp, h->s, sc, dial_mode, h->precision, st);
    } else {
        if (h->step_path == 2 && h->have_tiles)
            e = launch_tri_tiles(h->m, h->plan, h->s, sc, dial_mode, h->precision, st);
        else
            e = launch_tri_aos(h->m, h->plan, h->s, sc, dial_mode, h->precision, st);
        if (e == cudaSuccess) e = launch_node_update(h->m, h->s, sc, h->precision, st);
    }
    return e;
}

ms_status ms_set_step_path(ms_handle* h, int path) {
    if (!h || path < 0 || path > 4) return MS_ERR_INVALID_ARGUMENT;
    if (path == 0 && !h->have_cluster) return fail(h, MS_ERR_UNSUPPORTED, "cluster launches are unavailable");
    if (path == 2 && !h->have_tiles) return fail(h, MS_ERR_UNSUPPORTED, "bulk-copy tile kernel unavailable");
    if (path == 3 && !h->have_ntiles) return fail(h, MS_ERR_UNSUPPORTED, "node-tiled kernel unavailable");
    if (path == 4 && !h->have_pipe) return fail(h, MS_ERR_UNSUPPORTED, "warp-specialised node-tiled kernel unavailable");
    h->step_path = path;
    return MS_OK;
}

ms_status ms_step_n(ms_handle* h, int n, const double* dials, int dialling, double dt, double damping, int gd,
                    int check_last, ms_step_report* rep) {
    if (!h || n < 0) return MS_ERR_INVALID_ARGUMENT;
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->error_step = -1;
        rep->offending_dof = -1;
    }
    if (n == 0) return MS_OK;
    if (dialling && (!dials || !h->programmed))
        return fail(h, MS_ERR_INVALID_ARGUMENT, "dialling steps need dial factors and ms_set_programmed");
    const bool fuse_lce = dialling && lce_fusable(h);
    const int dial_mode = fuse_lce ? DIAL_LCE : DIAL_ARRAYS;
    const bool cluster = use_cluster(h, dialling != 0);
    cudaStream_t st = h->stream;
    // Steps that read abar/bbar from the arrays need them current; fused
    // protocol-3 steps dial in the kernel and leave them stale.
    if (!fuse_lce) MS_TRY(materialise_programmed(h));
    if (dialling) MS_TRY(stage_dials(h, dials, n));
    MS_TRY(reset_error(h));
    const int p0 = h->cur;
    int done = 0;
    while (done < n) {
        const int len = std::min(kChunk, n - done);
        const bool last_chunk = done + len == n;
        GraphKey key{len, p0 ^ (done & 1), dial_mode + (cluster ? 16 : 0) + 32 * h->step_path, gd,
                     (check_last && last_chunk) ? 1 : 0,
                     dt, damping};
        cudaGraphExec_t exec = nullptr;
        if (!(dialling && !fuse_lce))
            for (auto& g : h->graphs)
                if (g.key == key) {
                    exec = g.exec;
                    g.last_use = ++h->use_clock;
                }
        if (!exec) {
            // Non-LCE dialling materialises abar/bbar with the dialling kernel
            // each step; that kernel takes the dial factor by value, so those
            // segments are launched directly instead of through a graph.
            if (dialling && !fuse_lce) {
                for (int i = 0; i < len; ++i) {
                    MS_CUDA(h, launch_dialling(h->m, h->protocol, dials[done + i], h->spacing, h->from_ansatz, st));
                    StepScalars sc{i, key.parity ^ (i & 1), dt, damping, h->rho_hh, h->force_limit, gd,
                                   (key.check_last && i == len - 1) ? 1 : 0};
                    MS_CUDA(h, launch_step(h, sc, cluster, DIAL_ARRAYS, st));
                }
                MS_CUDA(h, launch_chunk_end(h->s, len, st));
                done += len;
                continue;
            }
            MS_TRY(capture_steps(h, key, cluster, &exec));
        }
        MS_CUDA(h, cudaGraphLaunch(exec, st));
        done += len;
    }
    MS_CUDA(h, cudaMemcpyAsync(h->h_err, h->s.err, sizeof(DevError), cudaMemcpyDeviceToHost, st));
    if (check_last) MS_CUDA(h, cudaMemcpyAsync(h->h_equil, h->s.equil, sizeof(DevEquil), cudaMemcpyDeviceToHost, st));
    MS_CUDA(h, cudaStreamSynchronize(st));
    if (h->h_err->flag) {
        const unsigned long long key = h->h_err->guard_key;
        const int step = (int)(key >> 32);
        const long long dof = (long long)(key & 0xffffffffULL);
        h->cur = p0 ^ (step & 1);
        // Recompute the failing step's forces from its saved input state, as
        // the reference holds them when it throws (main.cpp:448-474).
        if (dialling) {
            MS_CUDA(h, launch_dialling(h->m, h->protocol, dials[step], h->spacing, h->from_ansatz, st));
            h->ab_stale = false;
        }
        MS_CUDA(h, launch_surface_derivs(h->m, h->s, h->cur, st));
        MS_CUDA(h, launch_forces_from_cq(h->m, h->s, 0, st));
        MS_CUDA(h, launch_gather_forces(h->m, h->s, st));
        if (!gd) MS_CUDA(h, launch_damping(h->m, h->s, h->cur, damping, h->rho_hh, st));
        MS_CUDA(h, launch_constraints(h->m, h->s, st));
        double f = 0.0;
        MS_CUDA(h, cudaMemcpyAsync(&f, h->s.forces + dof, sizeof(double), cudaMemcpyDeviceToHost, st));
        MS_CUDA(h, cudaStreamSynchronize(st));
        if (rep) {
            rep->steps_done = step;
            rep->error_step = step;
            rep->offending_dof = dof;
            rep->offending_force = f;
        }
        return fail(h, MS_ERR_IMPLAUSIBLE_FORCE, "implausibly_high_force");
    }
    // The fused LCE path never wrote abar/bbar: they stand for the last
    // dialled step from here on and are formed when a call reads them.
    if (fuse_lce) {
        h->ab_stale = true;
        h->stale_dial = dials[n - 1];
    }
    h->cur = p0 ^ (n & 1);
    if (rep) {
        rep->steps_done = n;
        if (check_last) fill_equil(h, *h->h_equil, &rep->equil);
    }
    return MS_OK;
}

ms_status ms_prepare_steps(ms_handle* h, int n, int dialling, double dt, double damping, int gd, int check_last) {
    if (!h || n < 0) return MS_ERR_INVALID_ARGUMENT;
    if (n == 0) return MS_OK;
    if (dialling && !h->programmed)
        return fail(h, MS_ERR_INVALID_ARGUMENT, "dialling steps need ms_set_programmed");
    const bool fuse_lce = dialling && lce_fusable(h);
    if (dialling && !fuse_lce) return MS_OK;  // launched step by step, no graph to build
    const int dial_mode = fuse_lce ? DIAL_LCE : DIAL_ARRAYS;
    const bool cluster = use_cluster(h, dialling != 0);
    if (dialling) {
        // The dial-factor buffer the graphs read must be in place first.
        std::vector<double> zeros(n, 0.0);
        MS_TRY(stage_dials(h, zeros.data(), n));
        MS_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    const int p0 = h->cur;
    for (int done = 0; done < n;) {
        const int len = std::min(kChunk, n - done);
        GraphKey key{len, p0 ^ (done & 1), dial_mode + (cluster ? 16 : 0) + 32 * h->step_path, gd,
                     (check_last && done + len == n) ? 1 : 0, dt, damping};
        bool have = false;
        for (auto& g : h->graphs) have = have || g.key == key;
        if (!have) {
            cudaGraphExec_t exec;
            MS_TRY(capture_steps(h, key, cluster, &exec));
        }
        done += len;
    }
    return MS_OK;
}

void* ms_stream(ms_handle* h) { return h ? (void*)h->stream : nullptr; }

ms_status ms_time_kernels(ms_handle* h, int reps, int dialling, double dial, double dt, double damping, double* ms_tri,
                          double* ms_node) {
    if (!h || reps <= 0 || !ms_tri || !ms_node) return MS_ERR_INVALID_ARGUMENT;
    if (dialling && !h->programmed) return fail(h, MS_ERR_INVALID_ARGUMENT, "ms_set_programmed has not been called");
    const bool fuse_lce = dialling && lce_fusable(h);
    if (dialling && !fuse_lce) return fail(h, MS_ERR_UNSUPPORTED, "kernel timing covers the fused protocol-3 path");
    const bool cluster = use_cluster(h, dialling != 0);
    cudaStream_t st = h->stream;
    if (!fuse_lce) MS_TRY(materialise_programmed(h));
    if (dialling) {
        std::vector<double> d(reps, dial);
        MS_TRY(stage_dials(h, d.data(), reps));
    }
    MS_TRY(reset_error(h));
    std::vector<cudaEvent_t> ev(3 * reps);
    for (auto& e : ev) MS_CUDA(h, cudaEventCreate(&e));
    int p = h->cur;
    for (int i = 0; i < reps; ++i) {
        StepScalars sc{i, p, dt, damping, h->rho_hh, h->force_limit, 0, 0};
        const int mode = fuse_lce ? DIAL_LCE : DIAL_ARRAYS;
        MS_CUDA(h, cudaEventRecord(ev[3 * i], st));
        if (cluster) MS_CUDA(h, launch_cluster_step(h->m, h->plan, h->s, sc, mode, h->precision, st));
        else if (h->step_path == 4 && h->have_pipe)
            MS_CUDA(h, launch_node_pipe(h->m, h->plan, h->ntp, h->s, sc, mode, h->precision, st));
        else if (h->step_path == 3 && h->have_ntiles)
            MS_CUDA(h, launch_node_tiles(h->m, h->plan, h->ntp, h->s, sc, mode, h->precision, st));
        else if (h->step_path == 2 && h->have_tiles)
            MS_CUDA(h, launch_tri_tiles(h->m, h->plan, h->s, sc, mode, h->precision, st));
        else MS_CUDA(h, launch_tri_aos(h->m, h->plan, h->s, sc, mode, h->precision, st));
        MS_CUDA(h, cudaEventRecord(ev[3 * i + 1], st));
        if (cluster) MS_CUDA(h, launch_halo_update(h->m, h->plan, h->s, sc, h->precision, st));
        else if (!one_kernel_step(h)) MS_CUDA(h, launch_node_update(h->m, h->s, sc, h->precision, st));
        MS_CUDA(h, cudaEventRecord(ev[3 * i + 2], st));
        p ^= 1;
    }
    MS_CUDA(h, cudaStreamSynchronize(st));
    double a = 0, b = 0;
    for (int i = 0; i < reps; ++i) {
        float t1 = 0, t2 = 0;
        cudaEventElapsedTime(&t1, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&t2, ev[3 * i + 1], ev[3 * i + 2]);
        a += t1;
        b += t2;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    MS_CUDA(h, cudaMemcpy(h->h_err, h->s.err, sizeof(DevError), cudaMemcpyDeviceToHost));
    if (h->h_err->flag) return fail(h, MS_ERR_IMPLAUSIBLE_FORCE, "implausibly_high_force during kernel timing");
    h->cur = p;
    *ms_tri = a / reps;
    *ms_node = (!cluster && one_kernel_step(h)) ? 0.0 : b / reps;  // paths 3 and 4 have no node kernel
    return MS_OK;
}

ms_status ms_plan_info(ms_handle* h, int* cluster_size, int* tris_per_cta, int* clusters, int* halo_nodes,
                       int* path) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    if (cluster_size) *cluster_size = h->have_plan ? h->plan.cs : 0;
    if (tris_per_cta) *tris_per_cta = h->have_plan ? h->plan.tpc : 0;
    if (clusters) *clusters = h->have_plan ? h->plan.nclusters : 0;
    if (halo_nodes) *halo_nodes = h->have_plan ? h->plan.n_halo : -1;
    if (path) *path = h->have_plan ? h->step_path : 1;
    return MS_OK;
}

ms_status ms_node_tile_plan(ms_handle* h, int* nodes_per_tile, int* tiles, int* chunks, int* blocks) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    const bool ok = h->have_ntiles || h->have_pipe;
    const int grid = h->step_path == 4 ? h->ntp.grid_pipe : h->ntp.grid;
    if (nodes_per_tile) *nodes_per_tile = ok ? h->ntp.nodes : 0;
    if (tiles) *tiles = ok ? h->ntp.ntiles : 0;
    if (chunks) *chunks = ok ? h->ntp.nchunks : 0;
    if (blocks) *blocks = ok ? std::min(h->ntp.ntiles, grid) : 0;
    return MS_OK;
}

ms_status ms_node_tile_layout(int num_nodes, int num_tris, const int* patch_ids, int nodes_per_tile, int precision,
                              ms_node_tile_info* out) {
    if (num_nodes <= 0 || num_tris <= 0 || !patch_ids || !out) return MS_ERR_INVALID_ARGUMENT;
    const int N = num_nodes, T = num_tris;
    for (long long k = 0; k < 6LL * T; ++k)
        if (patch_ids[k] < 0 || patch_ids[k] >= N) return MS_ERR_INVALID_ARGUMENT;
    std::vector<int> off(N + 1, 0), ent(6ULL * T);
    for (long long k = 0; k < 6LL * T; ++k) off[patch_ids[k] + 1] += 1;
    for (int n = 0; n < N; ++n) off[n + 1] += off[n];
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 6; ++k) ent[fill[patch_ids[6LL * t + k]]++] = 6 * t + k;
    NodeTileLayout L;
    std::string err;
    if (!node_tile_layout(patch_ids, N, T, nodes_per_tile, precision == MS_PRECISION_MIXED, off, ent, L, err))
        return MS_ERR_INVALID_ARGUMENT;
    out->tiles = L.K;
    out->chunks = L.C;
    out->tri_tile_pairs = L.start[L.K];
    out->node_section_max = (long long)L.ns_max;
    out->record_stride = (long long)L.stride;
    long long b = 0;
    for (unsigned x : L.bytes) b += x;
    out->bytes_per_step = b;
    out->shared_bytes = (long long)node_tile_smem(L.stride, nodes_per_tile, precision == MS_PRECISION_MIXED);
    out->sliced_entries = L.slc_max;
    out->pipe_shared_bytes =
        (long long)node_pipe_smem(L.stride_sliced, nodes_per_tile, L.slc_max, precision == MS_PRECISION_MIXED);
    return MS_OK;
}

ms_status ms_output_quantities(ms_handle* h, double* curv, double* edens, double* strains, double* stresses,
                               double* deficits, double* energies) {
    if (!h) return MS_ERR_INVALID_ARGUMENT;
    const size_t T = h->m.T, N = h->m.N;
    cudaStream_t st = h->stream;
    MS_TRY(materialise_programmed(h));
    MS_CUDA(h, launch_surface_derivs(h->m, h->s, h->cur, st));
    MS_TRY(ensure_out(h, (2 * T + 2 * T + T + 8 * T + N) * sizeof(double)));
    double* dcurv = h->d_out;
    double* dedens = dcurv + 2 * T;
    double* dstrain = dedens + 2 * T;
    double* dstress = dstrain + T;
    double* ddef = dstress + 8 * T;
    MS_CUDA(h, launch_output_tri(h->m, h->s, dcurv, dedens, dstrain, dstress, h->d_scratch_tri, st));
    if (deficits) MS_CUDA(h, launch_angle_deficits(h->m, h->s, h->cur, ddef, st));
    if (energies) {
        MS_CUDA(h, launch_kinetic(h->m, h->s, h->cur, h->d_scratch_node, st));
        MS_CUDA(h, launch_comp_sum(h->d_scratch_tri, (int)T, h->d_sum_partial, h->d_sums + 0, st));
        MS_CUDA(h, launch_comp_sum(h->d_scratch_tri + T, (int)T, h->d_sum_partial, h->d_sums + 1, st));
        MS_CUDA(h, launch_comp_sum(h->d_scratch_node, (int)N, h->d_sum_partial, h->d_sums + 2, st));
        MS_CUDA(h, cudaMemcpyAsync(energies, h->d_sums, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (curv) MS_CUDA(h, cudaMemcpyAsync(curv, dcurv, 2 * T * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (edens) MS_CUDA(h, cudaMemcpyAsync(edens, dedens, 2 * T * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (strains) MS_CUDA(h, cudaMemcpyAsync(strains, dstrain, T * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (stresses) MS_CUDA(h, cudaMemcpyAsync(stresses, dstress, 8 * T * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (deficits) MS_CUDA(h, cudaMemcpyAsync(deficits, ddef, N * sizeof(double), cudaMemcpyDeviceToHost, st));
    MS_CUDA(h, cudaStreamSynchronize(st));
    return MS_OK;
}

}  // extern "C"
