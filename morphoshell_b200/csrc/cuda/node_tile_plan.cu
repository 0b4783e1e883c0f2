// Host side of the node-tiled step (node_tiles.cu, the batched variant in
// batch.cu): the layout of a plan (every tile's triangle list, its chunks and
// their node sections, checked against every bound the kernels rely on),
// the choice of tile size, and the chunk records themselves.
#include <algorithm>
#include <cstdlib>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

namespace msb {
namespace {

// Threads for the per-tile and per-chunk loops: MORPHOSHELL_SETUP_THREADS,
// else the hardware's; one for small plans.
int plan_threads(long long n) {
    if (n < 256) return 1;
    int t = (int)std::thread::hardware_concurrency();
    if (const char* e = std::getenv("MORPHOSHELL_SETUP_THREADS")) t = std::atoi(e);
    return std::max(1, std::min(t, 64));
}

// f(begin, end, worker) over [0, n) in contiguous ranges, one per thread;
// the first exception (of the lowest range) is rethrown after all joined.
template <typename F>
void parallel_ranges(int n, int threads, F f) {
    threads = std::max(1, std::min(threads, n));
    if (threads <= 1) {
        f(0, n, 0);
        return;
    }
    std::vector<std::thread> pool;
    std::vector<std::exception_ptr> errs(threads);
    const int chunk = (n + threads - 1) / threads;
    for (int w = 0; w < threads; ++w)
        pool.emplace_back([&, w]() {
            try {
                f(std::min(n, w * chunk), std::min(n, (w + 1) * chunk), w);
            } catch (...) {
                errs[w] = std::current_exception();
            }
        });
    for (auto& t : pool) t.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}

}  // namespace

bool node_tile_layout(const int* patch_ids, int N, int T, int NT, int mixed, const std::vector<int>& off,
                      const std::vector<int>& ent, NodeTileLayout& L, std::string& err, int sliced) {
    if (NT <= 0 || NT > kNtMaxNodes) {
        err = "nodes per tile must be in 1..32768";
        return false;
    }
    const int K = (N + NT - 1) / NT;
    L.K = K;
    L.start.assign(K + 1, 0);
    auto tiles_of = [&](int t, int* out) {
        int n = 0;
        for (int k = 0; k < 6; ++k) {
            const int tk = patch_ids[6LL * t + k] / NT;
            bool seen = false;
            for (int j = 0; j < n; ++j) seen = seen || out[j] == tk;
            if (!seen) out[n++] = tk;
        }
        return n;
    };
    int tk[6];
    for (int t = 0; t < T; ++t) {
        const int n = tiles_of(t, tk);
        for (int j = 0; j < n; ++j) L.start[tk[j] + 1] += 1;
    }
    for (int k = 0; k < K; ++k) L.start[k + 1] += L.start[k];
    L.lst.assign(L.start[K], 0);
    {
        std::vector<long long> fill(L.start.begin(), L.start.end() - 1);
        for (int t = 0; t < T; ++t) {
            const int n = tiles_of(t, tk);
            for (int j = 0; j < n; ++j) L.lst[fill[tk[j]]++] = t;
        }
    }
    L.tile_chunk.assign(K + 1, 0);
    // At least one chunk per tile (an empty one for a tile of isolated
    // nodes), so that every tile's walk starts with a copy of its own record.
    for (int k = 0; k < K; ++k)
        L.tile_chunk[k + 1] =
            L.tile_chunk[k] + std::max(1, (int)((L.start[k + 1] - L.start[k] + kTile - 1) / kTile));
    const int C = L.tile_chunk[K];
    L.C = C;
    // Node sections: for each chunk, runs (node in tile, end) and entries
    // (patch slot * 3 kTile + slot in chunk).  Nodes go in ascending order and each node's
    // entries in ascending t, so a node's entries within a chunk are one run.
    // A node's last run in its tile carries kRunFinal: once it is added the
    // node's force is complete.  A node with no entries gets an empty final
    // run in its tile's last chunk, so every node of a tile has exactly one.
    L.run_node.assign(C, {});
    L.run_end.assign(C, {});
    L.cent.assign(C, {});
    std::vector<int> run_last(C, -1);
    const int threads = plan_threads(C);
    std::vector<char> bad(threads, 0);
    // Each tile writes only its own chunks' lists: tiles in parallel.
    parallel_ranges(K, threads, [&](int k0, int k1, int w) {
        for (int k = k0; k < k1 && !bad[w]; ++k) {
            const int* L0 = L.lst.data() + L.start[k];
            const int* L1 = L.lst.data() + L.start[k + 1];
            for (int n = k * NT; n < std::min(N, (k + 1) * NT) && !bad[w]; ++n) {
                int last_t = -1, last_c = -1;
                if (off[n] == off[n + 1]) {
                    const int c = L.tile_chunk[k + 1] - 1;
                    L.run_node[c].push_back((unsigned short)((n - k * NT) | kRunFinal));
                    L.run_end[c].push_back(L.run_end[c].empty() ? 0 : L.run_end[c].back());
                    run_last[c] = n - k * NT;
                    continue;
                }
                for (int e = off[n]; e < off[n + 1]; ++e) {
                    const int t = ent[e] / 6, slot = ent[e] % 6;
                    const int li = (int)(std::lower_bound(L0, L1, t) - L0);
                    if (L0 + li == L1 || L0[li] != t || t < last_t) {
                        bad[w] = 1;
                        break;
                    }
                    last_t = t;
                    const int c = L.tile_chunk[k] + li / kTile;
                    const int j = n - k * NT;
                    if (run_last[c] != j) {
                        L.run_node[c].push_back((unsigned short)j);
                        L.run_end[c].push_back(L.run_end[c].empty() ? 0 : L.run_end[c].back());
                        run_last[c] = j;
                    }
                    L.cent[c].push_back((unsigned short)(slot * 3 * kTile + li % kTile));
                    L.run_end[c].back() += 1;
                    last_c = c;
                }
                if (!bad[w]) L.run_node[last_c].back() |= kRunFinal;
            }
        }
    });
    for (char b : bad)
        if (b) {
            err = "incidence lists disagree with the patches";
            return false;
        }
    // Within a chunk the runs are independent (distinct nodes), so their
    // order is free: longest first, so that the runs a warp takes together
    // (one per thread) have similar lengths and no lane waits long for
    // another.  Each run keeps its entries in ascending t.
    parallel_ranges(C, threads, [&](int c0, int c1, int) {
        std::vector<int> idx;
        std::vector<unsigned short> rn, re, ce;
        for (int c = c0; c < c1; ++c) {
            const int R = (int)L.run_node[c].size();
            idx.resize(R);
            for (int r = 0; r < R; ++r) idx[r] = r;
            auto len = [&](int r) { return (int)L.run_end[c][r] - (r ? (int)L.run_end[c][r - 1] : 0); };
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return len(a) > len(b); });
            rn.clear();
            re.clear();
            ce.clear();
            for (int r : idx) {
                const int e0 = r ? L.run_end[c][r - 1] : 0;
                for (int e = e0; e < (int)L.run_end[c][r]; ++e) ce.push_back(L.cent[c][e]);
                rn.push_back(L.run_node[c][r]);
                re.push_back((unsigned short)ce.size());
            }
            L.run_node[c].swap(rn);
            L.run_end[c].swap(re);
            L.cent[c].swap(ce);
        }
    });
    // The sliced order of each chunk's entries (the warp-specialised step):
    // slice s holds runs 32s .. 32s + 31, 32 entries per row, as many rows
    // as its first (longest) run has entries.
    L.slice_off.assign(C, {});
    L.dst.assign(C, {});
    std::vector<int> slc_w(threads, 32);
    std::fill(bad.begin(), bad.end(), 0);
    parallel_ranges(C, threads, [&](int c0, int c1, int w) {
        std::vector<unsigned char> used;
        for (int c = c0; c < c1 && !bad[w]; ++c) {
            const auto& re = L.run_end[c];
            const int R = (int)re.size();
            auto len = [&](int r) { return (int)re[r] - (r ? (int)re[r - 1] : 0); };
            std::vector<unsigned short>& so = L.slice_off[c];
            int off = 0;
            for (int r = 0; r < R; r += 32) {
                so.push_back((unsigned short)off);
                off += 32 * len(r);
            }
            if (off >= 65535) {
                bad[w] = 1;
                break;
            }
            slc_w[w] = std::max(slc_w[w], (off + 31) / 32 * 32);
            std::vector<unsigned short>& d = L.dst[c];
            d.assign(6 * kTile, 0xFFFF);
            // Every sliced position gets at most one contribution and lies
            // inside its slice (runs within a slice are no longer than its
            // first), so no two writes of a chunk collide.
            used.assign(off, 0);
            for (int r = 0; r < R && !bad[w]; ++r) {
                const int e0 = r ? re[r - 1] : 0;
                if (len(r) > len(r / 32 * 32)) {
                    bad[w] = 1;
                    break;
                }
                for (int e = e0; e < (int)re[r]; ++e) {
                    const int ce = L.cent[c][e], sl = ce / (3 * kTile), li = ce % (3 * kTile);
                    const int pos = so[r / 32] + 32 * (e - e0) + r % 32;
                    if (sl >= 6 || li >= kTile || pos >= off || used[pos] || d[sl * kTile + li] != 0xFFFF) {
                        bad[w] = 1;
                        break;
                    }
                    used[pos] = 1;
                    d[sl * kTile + li] = (unsigned short)pos;
                }
            }
        }
    });
    for (char b : bad)
        if (b) {
            err = "node tile chunk fails its bounds";
            return false;
        }
    L.slc_max = *std::max_element(slc_w.begin(), slc_w.end());
    L.fixed = tile_record_bytes(mixed);
    L.sliced = sliced != 0;
    size_t ns_max_sliced = 16;
    L.bytes.assign(C, 0);
    std::vector<size_t> ns_w(threads, 16), nss_w(threads, 16);
    std::fill(bad.begin(), bad.end(), 0);
    parallel_ranges(K, threads, [&](int k0, int k1, int w) {
        std::vector<unsigned char> finals;
        for (int k = k0; k < k1 && !bad[w]; ++k) {
            // Every node of the tile has exactly one final run.
            const int nn = std::min(N, (k + 1) * NT) - k * NT;
            finals.assign(nn, 0);
            for (int c = L.tile_chunk[k]; c < L.tile_chunk[k + 1]; ++c)
                for (unsigned short u : L.run_node[c])
                    if ((u & kRunFinal) && (u & ~kRunFinal) < nn) finals[u & ~kRunFinal] += 1;
            for (int j = 0; j < nn; ++j)
                if (finals[j] != 1) bad[w] = 1;
            for (int c = L.tile_chunk[k]; c < L.tile_chunk[k + 1] && !bad[w]; ++c) {
                const long long first = L.start[k] + (long long)(c - L.tile_chunk[k]) * kTile;
                const int ntri = (int)std::max<long long>(0, std::min<long long>(kTile, L.start[k + 1] - first));
                const size_t R = L.run_node[c].size(), E = L.cent[c].size();
                // What the kernels index: entries inside the chunk's live
                // slots, run nodes among the tile's nodes (so inside its
                // accumulators and the mesh), run ends ascending up to E,
                // everything inside one record.
                bool ok = R <= 6 * kTile + NT && E <= 6 * kTile;
                for (size_t r = 0; ok && r < R; ++r)
                    ok = (L.run_node[c][r] & ~kRunFinal) < nn && L.run_end[c][r] >= (r ? L.run_end[c][r - 1] : 0);
                ok = ok && (R == 0 ? E == 0 : L.run_end[c][R - 1] == E);
                for (size_t e = 0; ok && e < E; ++e)
                    ok = L.cent[c][e] / (3 * kTile) < 6 && L.cent[c][e] % (3 * kTile) < ntri;
                if (!ok) {
                    bad[w] = 1;
                    break;
                }
                const size_t S = L.slice_off[c].size();
                const size_t ns_plain = (16 + 4 * R + 2 * E + 15) / 16 * 16;
                const size_t ns_sliced = (16 + 4 * R + 2 * E + 2 * S + 2 * 6 * kTile + 15) / 16 * 16;
                const size_t ns = L.sliced ? ns_sliced : ns_plain;
                ns_w[w] = std::max(ns_w[w], ns);
                nss_w[w] = std::max(nss_w[w], ns_sliced);
                L.bytes[c] = (unsigned)(L.fixed + ns);
            }
        }
    });
    for (char b : bad)
        if (b) {
            err = "node tile chunk fails its bounds";
            return false;
        }
    L.ns_max = *std::max_element(ns_w.begin(), ns_w.end());
    ns_max_sliced = *std::max_element(nss_w.begin(), nss_w.end());
    L.stride = L.fixed + (L.ns_max + 127) / 128 * 128;
    L.stride_sliced = L.fixed + (ns_max_sliced + 127) / 128 * 128;
    return true;
}

bool choose_node_tiles(const int* patch_ids, int N, int T, int mixed, int sms, int target, int nt_max, int nt_min,
                       const std::vector<int>& off, const std::vector<int>& ent,
                       const std::function<size_t(const NodeTileLayout&, int)>& smem_for,
                       const std::function<int(size_t)>& blocks_for, NodeTileLayout& L, int& NT, int& blocks,
                       std::string& err, int sliced) {
    blocks = 0;
    for (int attempt = 0; attempt < 4; ++attempt) {
        const long long slots = (long long)std::max(sms, 1) * target;
        const long long k = std::max(1LL, (N + slots * nt_max - 1) / (slots * nt_max));
        NT = std::max(std::min(nt_max, nt_min), (int)((N + k * slots - 1) / (k * slots)));
        L = NodeTileLayout();
        if (!node_tile_layout(patch_ids, N, T, NT, mixed, off, ent, L, err, sliced)) return false;
        const size_t smem = smem_for(L, NT);
        blocks = smem > 227 * 1024 ? 0 : blocks_for(smem);
        if (blocks >= target) break;
        nt_max = nt_max * 7 / 8;
    }
    return true;
}

// Chunk c's node section (header, runs, entries and, for a sliced layout,
// the sliced order) at dst, which holds zeros.
void write_node_section(const NodeTileLayout& L, int c, int ntri, unsigned char* dst) {
    int32_t* hd = reinterpret_cast<int32_t*>(dst);
    const int R = (int)L.run_node[c].size(), E = (int)L.cent[c].size();
    const int S = L.sliced ? (int)L.slice_off[c].size() : 0;
    hd[0] = R;
    hd[1] = E;
    hd[2] = ntri;
    hd[3] = S;
    unsigned short* u = reinterpret_cast<unsigned short*>(dst + 16);
    std::copy(L.run_node[c].begin(), L.run_node[c].end(), u);
    std::copy(L.run_end[c].begin(), L.run_end[c].end(), u + R);
    std::copy(L.cent[c].begin(), L.cent[c].end(), u + 2 * R);
    if (L.sliced) {
        std::copy(L.slice_off[c].begin(), L.slice_off[c].end(), u + 2 * R + E);
        std::copy(L.dst[c].begin(), L.dst[c].end(), u + 2 * R + E + S);
    }
}

// Live triangles of chunk c of tile k.
static int chunk_live(const NodeTileLayout& L, int k, int c) {
    const long long first = L.start[k] + (long long)(c - L.tile_chunk[k]) * kTile;
    return (int)std::max<long long>(0, std::min<long long>(kTile, L.start[k + 1] - first));
}

void fill_node_tile_records(const NodeTileLayout& L, const int* patch_ids, const double* coef_d, const float* coef_f,
                            const double* area, const double* aux4, int mixed, std::vector<unsigned char>& buf,
                            std::vector<int>& chunk_tri) {
    const size_t stride = L.stride, fixed = L.fixed;
    buf.assign(stride * L.C, 0);
    chunk_tri.assign((size_t)L.C * kTile, -1);
    const size_t ids_b = 6 * kTile * 4, coef_b = 24 * kTile * (mixed ? 4 : 8);
    parallel_ranges(L.K, plan_threads(L.C), [&](int k0, int k1, int) {
        for (int k = k0; k < k1; ++k) {
            for (int c = L.tile_chunk[k]; c < L.tile_chunk[k + 1]; ++c) {
                unsigned char* r = buf.data() + stride * c;
                int32_t* ids = reinterpret_cast<int32_t*>(r);
                double* aux = reinterpret_cast<double*>(r + ids_b + coef_b);
                const long long first = L.start[k] + (long long)(c - L.tile_chunk[k]) * kTile;
                const int ntri = chunk_live(L, k, c);
                for (int i = 0; i < ntri; ++i) {
                    const int t = L.lst[first + i];
                    chunk_tri[(size_t)c * kTile + i] = t;
                    for (int q = 0; q < 6; ++q) ids[q * kTile + i] = patch_ids[6LL * t + q];
                    if (mixed) {
                        float* cf = reinterpret_cast<float*>(r + ids_b);
                        for (int q = 0; q < 24; ++q)
                            cf[q * kTile + i] = coef_f ? coef_f[24LL * t + q] : (float)coef_d[24LL * t + q];
                    } else {
                        double* cf = reinterpret_cast<double*>(r + ids_b);
                        for (int q = 0; q < 24; ++q) cf[q * kTile + i] = coef_d[24LL * t + q];
                    }
                    if (aux4) {
                        for (int q = 0; q < 4; ++q) aux[q * kTile + i] = aux4[4LL * t + q];
                    } else {
                        aux[i] = area[t];
                        aux[kTile + i] = 1.0;
                    }
                }
                write_node_section(L, c, ntri, r + fixed);
            }
        }
    });
}

void fill_node_sections(const NodeTileLayout& L, size_t pitch, std::vector<unsigned char>& sections,
                        std::vector<int>& chunk_tri) {
    sections.assign(pitch * L.C, 0);
    chunk_tri.assign((size_t)L.C * kTile, -1);
    parallel_ranges(L.K, plan_threads(L.C), [&](int k0, int k1, int) {
        for (int k = k0; k < k1; ++k)
            for (int c = L.tile_chunk[k]; c < L.tile_chunk[k + 1]; ++c) {
                const long long first = L.start[k] + (long long)(c - L.tile_chunk[k]) * kTile;
                const int ntri = chunk_live(L, k, c);
                for (int i = 0; i < ntri; ++i) chunk_tri[(size_t)c * kTile + i] = L.lst[first + i];
                write_node_section(L, c, ntri, sections.data() + pitch * c);
            }
    });
}

}  // namespace msb
