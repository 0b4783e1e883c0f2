// Deformation forces without any device allocation (ms_deformation_forces_noalloc
// in include/morphoshell_gpu.h).
//
// Who needs it: callers that cannot call cudaMalloc -- host frameworks that
// route every device allocation through their own pool and forbid others
// (an allocation behind the pool's back breaks its accounting and can fail
// once the pool holds the memory), and real-time loops that must not
// allocate after start-up (cudaMalloc can block on the device and take
// unbounded time).  They already hold device buffers for the mesh tables, the
// positions and the forces; this entry point computes forces = -D^T dE/dcq
// from them using a fixed scratch area that lives in this library's static
// device memory.
//
// Scratch: one file-scope __device__ array sized for meshes of up to
// kMaxTris triangles and kMaxNodes nodes (about 11.5 MB, held by every GPU
// that loads the library until the process exits).  Larger meshes are
// rejected.  Every call shares the array and it keeps the last call's
// contents, so two calls that overlap on the GPU (different streams, or
// different host threads on the same device) race and corrupt each other;
// serialise them.  The per-node counters are cleared at the start of every
// call.
//
// The node sums are deterministic: each node's incidence list is rebuilt in
// the scratch (integer counting, then each list sorted by triangle), and its
// contributions are added in ascending triangle order, as in the main path.
#include <cstdio>
#include <cstring>

#include "../../../include/morphoshell_gpu.h"
#include "tri_physics.cuh"

namespace {

constexpr int kMaxTris = 65536;
constexpr int kMaxNodes = 65536;

struct Scratch {
    double contrib[kMaxTris * 18];  // per (triangle, slot) force contribution
    int count[kMaxNodes + 1];       // entries per node, then exclusive offsets
    int cursor[kMaxNodes];          // fill cursors
    int entries[kMaxTris * 6];      // (6 t + slot) grouped by node
    int bad;                        // patch ids outside [0, num_nodes) seen this call
};

static __device__ __align__(256) unsigned char ms_noalloc_scratch[sizeof(Scratch)];

// Device address of the scratch array in the current context, looked up on
// every call (a table lookup once the module is loaded), so that an address
// never outlives the context it belongs to, e.g. across cudaDeviceReset.
cudaError_t scratch_address(Scratch** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, ms_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<Scratch*>(p);
    return cudaSuccess;
}

__global__ void k_na_zero(Scratch* s, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) s->count[i] = 0;
    if (i < n) s->cursor[i] = 0;
    if (i == 0) s->bad = 0;
}

// Ids outside [0, n) are counted as bad and skipped by every later kernel.
__global__ void k_na_count(Scratch* s, const int* __restrict__ patch, int T, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 6 * T) return;
    const int id = patch[k];
    if (id < 0 || id >= n) {
        atomicAdd(&s->bad, 1);
        return;
    }
    atomicAdd(&s->count[id + 1], 1);
}

// Inclusive scan of count[1..n] in place (one block): count[i] becomes the
// offset of node i's first entry.
__global__ void k_na_scan(Scratch* s, int n) {
    __shared__ int partial[1024];
    const int per = (n + 1 + blockDim.x - 1) / blockDim.x;
    const int lo = threadIdx.x * per, hi = min(n + 1, lo + per);
    int acc = 0;
    for (int i = lo; i < hi; ++i) acc += s->count[i];
    partial[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < (int)blockDim.x; ++w) {
            const int v = partial[w];
            partial[w] = run;
            run += v;
        }
    }
    __syncthreads();
    int run = partial[threadIdx.x];
    for (int i = lo; i < hi; ++i) {
        run += s->count[i];
        s->count[i] = run;
    }
}

__global__ void k_na_fill(Scratch* s, const int* __restrict__ patch, int T, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 6 * T) return;
    const int node = patch[k];
    if (node < 0 || node >= n) return;
    const int pos = s->count[node] + atomicAdd(&s->cursor[node], 1);
    s->entries[pos] = k;
}

// The fill order within a node depends on scheduling; sorting each short
// list makes the summation order the ascending-triangle order.
__global__ void k_na_sort(Scratch* s, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int* e = s->entries + s->count[i];
    const int len = s->count[i + 1] - s->count[i];
    for (int a = 1; a < len; ++a) {
        const int v = e[a];
        int b = a - 1;
        while (b >= 0 && e[b] > v) {
            e[b + 1] = e[b];
            --b;
        }
        e[b + 1] = v;
    }
}

__global__ void k_na_tri(Scratch* s, int N, int T, const int* __restrict__ patch, const double* __restrict__ coef,
                         const double* __restrict__ area, const double* __restrict__ thick,
                         const double* __restrict__ shear, const double* __restrict__ abar,
                         const double* __restrict__ bbar, double nu, double gamma, const double* __restrict__ dofs) {
    using namespace msb::dev;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    double c[24], P[6][3];
    for (int k = 0; k < 24; ++k) c[k] = coef[24 * (size_t)t + k];
    for (int k = 0; k < 6; ++k) {
        int id = patch[6 * (size_t)t + k];
        if (id < 0 || id >= N) id = 0;  // reported through Scratch::bad; never read out of range
        P[k][0] = dofs[id];
        P[k][1] = dofs[(size_t)N + id];
        P[k][2] = dofs[2 * (size_t)N + id];
    }
    double rx[3], ry[3], rxx[3], rxy[3], ryy[3];
    for (int i = 0; i < 3; ++i) {
        rx[i] = c[0] * P[0][i] + c[1] * P[1][i] + c[2] * P[2][i];
        ry[i] = c[3] * P[0][i] + c[4] * P[1][i] + c[5] * P[2][i];
        double sxx = 0, sxy = 0, syy = 0;
        for (int k = 0; k < 6; ++k) {
            sxx += c[6 + 3 * k] * P[k][i];
            sxy += c[7 + 3 * k] * P[k][i];
            syy += c[8 + 3 * k] * P[k][i];
        }
        rxx[i] = sxx;
        rxy[i] = sxy;
        ryy[i] = syy;
    }
    Cq<double> q;
    q.rx = {rx[0], rx[1], rx[2]};
    q.ry = {ry[0], ry[1], ry[2]};
    q.rxx = {rxx[0], rxx[1], rxx[2]};
    q.rxy = {rxy[0], rxy[1], rxy[2]};
    q.ryy = {ryy[0], ryy[1], ryy[2]};
    TriMat<double> m;
    m.abar0 = abar[3 * (size_t)t];
    m.abar1 = abar[3 * (size_t)t + 1];
    m.abar2 = abar[3 * (size_t)t + 2];
    m.bbar0 = bbar[3 * (size_t)t];
    m.bbar1 = bbar[3 * (size_t)t + 1];
    m.bbar2 = bbar[3 * (size_t)t + 2];
    m.h = thick[t];
    m.mu = shear[t];
    material_coefs(m.h, m.mu, nu, gamma, m.ks, m.kb, m.igmh);
    m.area = area[t];
    CqGrad<double> g;
    energy_gradient<double>(q, m, nu, g);
    double* o = s->contrib + 18 * (size_t)t;
    for (int k = 0; k < 6; ++k) {
        const double mxx = c[6 + 3 * k], mxy = c[7 + 3 * k], myy = c[8 + 3 * k];
        double fx = mxx * g.rxx.x + mxy * g.rxy.x + myy * g.ryy.x;
        double fy = mxx * g.rxx.y + mxy * g.rxy.y + myy * g.ryy.y;
        double fz = mxx * g.rxx.z + mxy * g.rxy.z + myy * g.ryy.z;
        if (k < 3) {
            fx += c[k] * g.rx.x + c[3 + k] * g.ry.x;
            fy += c[k] * g.rx.y + c[3 + k] * g.ry.y;
            fz += c[k] * g.rx.z + c[3 + k] * g.ry.z;
        }
        o[3 * k] = -fx;
        o[3 * k + 1] = -fy;
        o[3 * k + 2] = -fz;
    }
}

__global__ void k_na_gather(const Scratch* s, int N, double* __restrict__ forces) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int k = s->count[n]; k < s->count[n + 1]; ++k) {
        const double* c = s->contrib + 3 * (size_t)s->entries[k];
        fx += c[0];
        fy += c[1];
        fz += c[2];
    }
    forces[n] = fx;
    forces[(size_t)N + n] = fy;
    forces[2 * (size_t)N + n] = fz;
}

void set_msg(char* err, size_t len, const char* msg) {
    if (err && len) {
        std::strncpy(err, msg, len - 1);
        err[len - 1] = 0;
    }
}

}  // namespace

extern "C" ms_status ms_deformation_forces_noalloc(int32_t num_nodes, int32_t num_tris, const int32_t* patch_ids,
                                                   const double* deriv_coeffs, const double* ref_area,
                                                   const double* ref_thickness, const double* ref_shear_modulus,
                                                   const double* abar, const double* bbar, double def_poisson_ratio,
                                                   double bend_stiffening_scale_factor, const double* dofs,
                                                   double* forces, void* stream, char* err, size_t err_len) {
    set_msg(err, err_len, "");
    if (num_nodes <= 0 || num_tris <= 0 || !patch_ids || !deriv_coeffs || !ref_area || !ref_thickness ||
        !ref_shear_modulus || !abar || !bbar || !dofs || !forces) {
        set_msg(err, err_len, "ms_deformation_forces_noalloc: null pointer or non-positive size");
        return MS_ERR_INVALID_ARGUMENT;
    }
    if (num_tris > kMaxTris || num_nodes > kMaxNodes) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "ms_deformation_forces_noalloc: mesh of %d nodes / %d triangles exceeds the static scratch "
                      "limit of %d nodes / %d triangles",
                      (int)num_nodes, (int)num_tris, kMaxNodes, kMaxTris);
        set_msg(err, err_len, buf);
        return MS_ERR_INVALID_ARGUMENT;
    }
    Scratch* s = nullptr;
    cudaError_t e = scratch_address(&s);
    if (e != cudaSuccess) {
        set_msg(err, err_len, cudaGetErrorString(e));
        return e == cudaErrorNoDevice ? MS_ERR_NO_DEVICE : MS_ERR_CUDA;
    }
    // An error left pending by the caller's earlier work is not this call's:
    // report it without clearing it, and launch nothing.
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        char buf[200];
        std::snprintf(buf, sizeof buf, "ms_deformation_forces_noalloc: a CUDA error was pending before the call (%s)",
                      cudaGetErrorString(e));
        set_msg(err, err_len, buf);
        return MS_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int N = num_nodes, T = num_tris;
    // Each launch is checked on its own so the message names the kernel that
    // failed; the error is ours, so it is cleared.
    auto launched = [&](const char* name) -> bool {
        const cudaError_t le = cudaGetLastError();
        if (le == cudaSuccess) return true;
        char buf[200];
        std::snprintf(buf, sizeof buf, "ms_deformation_forces_noalloc: launch of %s failed (%s)", name,
                      cudaGetErrorString(le));
        set_msg(err, err_len, buf);
        return false;
    };
    k_na_zero<<<(N + 256) / 256, 256, 0, st>>>(s, N);
    if (!launched("k_na_zero")) return MS_ERR_CUDA;
    k_na_count<<<(6 * T + 255) / 256, 256, 0, st>>>(s, patch_ids, T, N);
    if (!launched("k_na_count")) return MS_ERR_CUDA;
    k_na_scan<<<1, 1024, 0, st>>>(s, N);
    if (!launched("k_na_scan")) return MS_ERR_CUDA;
    k_na_fill<<<(6 * T + 255) / 256, 256, 0, st>>>(s, patch_ids, T, N);
    if (!launched("k_na_fill")) return MS_ERR_CUDA;
    k_na_sort<<<(N + 255) / 256, 256, 0, st>>>(s, N);
    if (!launched("k_na_sort")) return MS_ERR_CUDA;
    k_na_tri<<<(T + 127) / 128, 128, 0, st>>>(s, N, T, patch_ids, deriv_coeffs, ref_area, ref_thickness,
                                               ref_shear_modulus, abar, bbar, def_poisson_ratio,
                                               bend_stiffening_scale_factor, dofs);
    if (!launched("k_na_tri")) return MS_ERR_CUDA;
    k_na_gather<<<(N + 255) / 256, 256, 0, st>>>(s, N, forces);
    if (!launched("k_na_gather")) return MS_ERR_CUDA;
    // Wait for the result and check the ids (a plain host int: no allocation).
    int bad = 0;
    e = cudaMemcpyAsync(&bad, &s->bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_msg(err, err_len, cudaGetErrorString(e));
        return MS_ERR_CUDA;
    }
    if (bad) {
        set_msg(err, err_len, "ms_deformation_forces_noalloc: patch ids outside [0, num_nodes); forces incomplete");
        return MS_ERR_INVALID_ARGUMENT;
    }
    return MS_OK;
}
