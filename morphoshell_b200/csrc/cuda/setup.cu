// Patch search, patch fit and derivative weights of every triangle on the
// device (set_up_patch_fitting.cpp:48-305, calc_deriv_mats.cpp:46-136): one
// thread per triangle, the host set-up's choices and arithmetic
// (patch_fit.hpp; this file compiles with -fmad=false, so each operation
// rounds as on the host).  The candidate order is the ascending distance
// order; where two candidate distances of a triangle are equal, the order
// std::sort gives them is the host's to decide, so that triangle (and any
// whose search does not finish here) is redone on the host.
#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../host/host.hpp"
#include "../host/patch_fit.hpp"

namespace msb {
namespace {

constexpr int kMaxCand = 64;

enum PatchStatus { PATCH_OK = 0, PATCH_TIE = 1, PATCH_OVERFLOW = 2, PATCH_FEW = 3, PATCH_NONE = 4 };

__global__ void k_patch_fit(int T, const double* __restrict__ P, const int* __restrict__ tv,
                            const double* __restrict__ cen, const unsigned char* __restrict__ boundary,
                            const int* __restrict__ inc_off, const int* __restrict__ inc_tri, double thresh,
                            int* __restrict__ extra, double* __restrict__ coeffs, int* __restrict__ status,
                            int* __restrict__ retries) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int v[3] = {tv[3 * (size_t)t], tv[3 * (size_t)t + 1], tv[3 * (size_t)t + 2]};
    const double c[3] = {cen[3 * (size_t)t], cen[3 * (size_t)t + 1], cen[3 * (size_t)t + 2]};
    retries[t] = 0;
    // Candidates: vertices of the triangles incident on the vertices, in the
    // host's visiting order, each once, the triangle's own vertices left out.
    int cand[kMaxCand];
    double dist[kMaxCand];
    int nc = 0;
    for (int a = 0; a < 3; ++a)
        for (int e = inc_off[v[a]]; e < inc_off[v[a] + 1]; ++e) {
            const int it = inc_tri[e];
            for (int w = 0; w < 3; ++w) {
                const int id = tv[3 * (size_t)it + w];
                bool seen = id == v[0] || id == v[1] || id == v[2];
                for (int k = 0; k < nc && !seen; ++k) seen = cand[k] == id;
                if (seen) continue;
                if (nc == kMaxCand) {
                    status[t] = PATCH_OVERFLOW;
                    return;
                }
                dist[nc] = patch::centroid_distance(P + 3 * (size_t)id, c);
                cand[nc++] = id;
            }
        }
    if (nc < 3) {
        status[t] = PATCH_FEW;
        return;
    }
    int ord[kMaxCand];
    for (int k = 0; k < nc; ++k) {
        int j = k;
        while (j > 0 && dist[ord[j - 1]] > dist[k]) {
            ord[j] = ord[j - 1];
            --j;
        }
        ord[j] = k;
    }
    for (int k = 0; k + 1 < nc; ++k)
        if (dist[ord[k]] == dist[ord[k + 1]]) {
            status[t] = PATCH_TIE;
            return;
        }
    double pos[6][3];
    for (int n = 0; n < 3; ++n)
        for (int k = 0; k < 3; ++k) pos[n][k] = P[3 * (size_t)v[n] + k];
    const int e0 = cand[ord[0]];
    for (int k = 0; k < 3; ++k) pos[3][k] = P[3 * (size_t)e0 + k];
    int nret = 0;
    const int pmax = nc < 4 ? nc : 4;
    for (int p = 1; p < pmax; ++p) {
        const int e1 = cand[ord[p]];
        for (int k = 0; k < 3; ++k) pos[4][k] = P[3 * (size_t)e1 + k];
        for (int q = 2; q < nc; ++q) {
            const int e2 = cand[ord[q]];
            for (int k = 0; k < 3; ++k) pos[5][k] = P[3 * (size_t)e2 + k];
            double block[6][3];
            if (!patch::try_patch(pos, c, thresh, block)) {
                if (q == 2 && !boundary[t]) ++nret;
                continue;
            }
            double* w = coeffs + 24 * (size_t)t;
            const double vpos[3][3] = {{pos[0][0], pos[0][1], pos[0][2]},
                                       {pos[1][0], pos[1][1], pos[1][2]},
                                       {pos[2][0], pos[2][1], pos[2][2]}};
            patch::first_derivative_weights(vpos, c, w);
            for (int n = 0; n < 6; ++n)
                for (int k = 0; k < 3; ++k) w[6 + 3 * n + k] = block[n][k];
            extra[3 * (size_t)t] = e0;
            extra[3 * (size_t)t + 1] = e1;
            extra[3 * (size_t)t + 2] = e2;
            retries[t] = nret;
            status[t] = PATCH_OK;
            return;
        }
    }
    status[t] = PATCH_NONE;
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("device set-up: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace

void set_up_patches_on_device(const std::vector<Node>& nodes, const DMat& P, std::vector<Tri>& triangles,
                              const Stuff& stuff, std::vector<double>& coeffs, Log& log) {
    const int N = (int)nodes.size(), T = (int)triangles.size();
    coeffs.assign(static_cast<size_t>(T) * 24, 0.0);
    if (T == 0) return;
    std::vector<int> tv(3ULL * T), inc_off(N + 1, 0), inc_tri;
    std::vector<double> cen(3ULL * T);
    std::vector<unsigned char> bnd(T);
    for (int t = 0; t < T; ++t) {
        const Tri& tri = triangles[t];
        for (int k = 0; k < 3; ++k) {
            tv[3ULL * t + k] = tri.vertex_ids[k];
            cen[3ULL * t + k] = tri.ref_centroid[k];
        }
        bnd[t] = tri.is_boundary ? 1 : 0;
    }
    for (int n = 0; n < N; ++n) inc_off[n + 1] = inc_off[n] + (int)nodes[n].incident_tri_ids.size();
    inc_tri.reserve(inc_off[N]);
    for (int n = 0; n < N; ++n)
        inc_tri.insert(inc_tri.end(), nodes[n].incident_tri_ids.begin(), nodes[n].incident_tri_ids.end());
    double *d_P = nullptr, *d_cen = nullptr, *d_coef = nullptr;
    int *d_tv = nullptr, *d_off = nullptr, *d_inc = nullptr, *d_extra = nullptr, *d_status = nullptr,
        *d_ret = nullptr;
    unsigned char* d_bnd = nullptr;
    std::vector<void*> allocs;
    auto dal = [&](void** p, size_t bytes) {
        check(cudaMalloc(p, std::max<size_t>(bytes, 1)), "cudaMalloc");
        allocs.push_back(*p);
    };
    std::vector<int> extra(3ULL * T), status(T), ret(T);
    std::vector<double> dev_coef(static_cast<size_t>(T) * 24);
    try {
        dal((void**)&d_P, sizeof(double) * P.v.size());
        dal((void**)&d_cen, sizeof(double) * cen.size());
        dal((void**)&d_coef, sizeof(double) * dev_coef.size());
        dal((void**)&d_tv, sizeof(int) * tv.size());
        dal((void**)&d_off, sizeof(int) * inc_off.size());
        dal((void**)&d_inc, sizeof(int) * inc_tri.size());
        dal((void**)&d_extra, sizeof(int) * extra.size());
        dal((void**)&d_status, sizeof(int) * status.size());
        dal((void**)&d_ret, sizeof(int) * ret.size());
        dal((void**)&d_bnd, bnd.size());
        check(cudaMemcpy(d_P, P.v.data(), sizeof(double) * P.v.size(), cudaMemcpyHostToDevice), "upload");
        check(cudaMemcpy(d_cen, cen.data(), sizeof(double) * cen.size(), cudaMemcpyHostToDevice), "upload");
        check(cudaMemcpy(d_tv, tv.data(), sizeof(int) * tv.size(), cudaMemcpyHostToDevice), "upload");
        check(cudaMemcpy(d_off, inc_off.data(), sizeof(int) * inc_off.size(), cudaMemcpyHostToDevice), "upload");
        if (!inc_tri.empty())
            check(cudaMemcpy(d_inc, inc_tri.data(), sizeof(int) * inc_tri.size(), cudaMemcpyHostToDevice), "upload");
        check(cudaMemcpy(d_bnd, bnd.data(), bnd.size(), cudaMemcpyHostToDevice), "upload");
        k_patch_fit<<<(T + 127) / 128, 128>>>(T, d_P, d_tv, d_cen, d_bnd, d_off, d_inc,
                                              stuff.patch_mat_dimless_conditioning_thresh, d_extra, d_coef,
                                              d_status, d_ret);
        check(cudaGetLastError(), "k_patch_fit launch");
        check(cudaMemcpy(dev_coef.data(), d_coef, sizeof(double) * dev_coef.size(), cudaMemcpyDeviceToHost),
              "download");
        check(cudaMemcpy(extra.data(), d_extra, sizeof(int) * extra.size(), cudaMemcpyDeviceToHost), "download");
        check(cudaMemcpy(status.data(), d_status, sizeof(int) * status.size(), cudaMemcpyDeviceToHost), "download");
        check(cudaMemcpy(ret.data(), d_ret, sizeof(int) * ret.size(), cudaMemcpyDeviceToHost), "download");
    } catch (...) {
        for (void* p : allocs) cudaFree(p);
        throw;
    }
    for (void* p : allocs) cudaFree(p);
    int num_interior_retries = 0;
    for (int t = 0; t < T; ++t) {
        Tri& tri = triangles[t];
        double* w = &coeffs[static_cast<size_t>(tri.id) * 24];
        if (status[t] == PATCH_OK) {
            const double* d = &dev_coef[static_cast<size_t>(t) * 24];
            std::copy(d, d + 24, w);
            for (int k = 0; k < 3; ++k) tri.non_vertex_patch_nodes_ids[k] = extra[3ULL * t + k];
            for (int n = 0; n < 6; ++n)
                for (int k = 0; k < 3; ++k) tri.mat_for_patch_2nd_derivs[n][k] = d[6 + 3 * n + k];
            num_interior_retries += ret[t];
        } else {
            // The host's search for this one (it throws as the host set-up
            // does when no patch passes).
            fit_patch(t, nodes, P, triangles, stuff.patch_mat_dimless_conditioning_thresh, num_interior_retries);
            deriv_coeffs_of(tri, P, w);
        }
    }
    log_patch_retries(log, num_interior_retries);
}

}  // namespace msb
