// Device self-checks of the reciprocal quotients of the FP64 right-hand side,
// built into lib/libgrt_selftest.so (test infrastructure; the product library
// does not link it), with -fmad=false like the trace kernels.
//   grt_selftest_division  div_by(a, b, RN(1/b)) and IEEE a / b on the same operands;
//   grt_selftest_rhs       ks_rhs_rcp (and its box flag) and ks_rhs on the same states;
//   grt_selftest_pow_quarter  the RK45 controller's pow_quarter on the device;
//   grt_selftest_rn_box    the branch-free reciprocal and square root (grt_rn.cuh)
//                          and CUDA's __drcp_rn and sqrt on the same arguments;
//   grt_selftest_rhs_bf    ks_rhs_rcp with the branch-free functions and with CUDA's.
#include <cuda_runtime.h>
#include <stdint.h>

#include "grt_metric.cuh"
#include "grt_pow_quarter.cuh"

namespace {

__global__ void division_kernel(const double* a, const double* b, size_t n, double* q_rcp, double* q_ieee) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    q_rcp[i] = grt::dev::div_by(a[i], b[i], grt::dev::div_recip(b[i]));
    q_ieee[i] = a[i] / b[i];
}

__global__ void rhs_kernel(const double* st, size_t n, double spin, double M, double* fast, double* ieee,
                           uint32_t* inside) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double* s = st + 7 * i;
    bool ok = false;
    const grt::dev::Rhs7 o = grt::dev::ks_rhs_rcp(s[0], s[1], s[2], s[3], s[4], s[5], s[6], spin, M, ok);
    const grt::dev::Rhs7 w = grt::dev::ks_rhs(s[0], s[1], s[2], s[3], s[4], s[5], s[6], spin, M);
    const double ov[7] = {o.t, o.x, o.y, o.z, o.px, o.py, o.pz};
    const double wv[7] = {w.t, w.x, w.y, w.z, w.px, w.py, w.pz};
    for (int c = 0; c < 7; ++c) {
        fast[7 * i + c] = ov[c];
        ieee[7 * i + c] = wv[c];
    }
    inside[i] = ok ? 1u : 0u;
}

__global__ void rn_box_kernel(const double* x, size_t n, double* rb, double* rc, double* sb, double* sc) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double v = fabs(x[i]);
    rb[i] = grt::dev::rcp_rn_box(x[i]);
    rc[i] = __drcp_rn(x[i]);
    sb[i] = grt::dev::sqrt_rn_box(v);
    sc[i] = sqrt(v);
}

__global__ void rhs_bf_kernel(const double* st, size_t n, double spin, double M, double* bf, double* ref,
                              uint32_t* inside) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double* s = st + 7 * i;
    bool ok_bf = false, ok_ref = false;
    const grt::dev::Rhs7 o = grt::dev::ks_rhs_rcp<true>(s[0], s[1], s[2], s[3], s[4], s[5], s[6], spin, M, ok_bf);
    const grt::dev::Rhs7 w = grt::dev::ks_rhs_rcp<false>(s[0], s[1], s[2], s[3], s[4], s[5], s[6], spin, M, ok_ref);
    const double ov[7] = {o.t, o.x, o.y, o.z, o.px, o.py, o.pz};
    const double wv[7] = {w.t, w.x, w.y, w.z, w.px, w.py, w.pz};
    for (int c = 0; c < 7; ++c) {
        bf[7 * i + c] = ov[c];
        ref[7 * i + c] = wv[c];
    }
    inside[i] = (ok_bf ? 1u : 0u) | (ok_ref ? 2u : 0u);
}

__global__ void pow_quarter_kernel(const double* x, size_t n, double* y) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    y[i] = grt::pow_quarter(x[i]);
}

template <int N>
struct Bufs {
    void* p[N] = {};
    int k = 0;
    ~Bufs() {
        for (int q = 0; q < k; ++q) cudaFree(p[q]);
    }
    template <class T>
    cudaError_t get(T** out, size_t count) {
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(out), count * sizeof(T) + 16);
        if (e == cudaSuccess) p[k++] = *out;
        return e;
    }
};

#define CK(x)                                  \
    do {                                       \
        cudaError_t e_ = (x);                  \
        if (e_ != cudaSuccess) return (int)e_; \
    } while (0)

}  // namespace

extern "C" {

// q_rcp[i] = div_by(a[i], b[i], RN(1/b[i])), q_ieee[i] = a[i] / b[i]; host
// arrays of n values.  Returns a cudaError_t.
int grt_selftest_division(const double* a, const double* b, size_t n, double* q_rcp, double* q_ieee) {
    if (n == 0) return 0;
    Bufs<4> B;
    double *da, *db, *dq, *dw;
    CK(B.get(&da, n));
    CK(B.get(&db, n));
    CK(B.get(&dq, n));
    CK(B.get(&dw, n));
    CK(cudaMemcpy(da, a, n * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(db, b, n * 8, cudaMemcpyHostToDevice));
    division_kernel<<<static_cast<unsigned>((n + 255) / 256), 256>>>(da, db, n, dq, dw);
    CK(cudaGetLastError());
    CK(cudaMemcpy(q_rcp, dq, n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(q_ieee, dw, n * 8, cudaMemcpyDeviceToHost));
    return 0;
}

// states[i] = (x, y, z, p_t, p_x, p_y, p_z); fast / ieee receive the seven
// right-hand-side components of ks_rhs_rcp / ks_rhs, inside[i] whether the
// state was in ks_rhs_rcp's box.
int grt_selftest_rhs(const double* states, size_t n, double spin, double M, double* fast, double* ieee,
                     uint32_t* inside) {
    if (n == 0) return 0;
    Bufs<4> B;
    double *ds, *df, *dw;
    uint32_t* din;
    CK(B.get(&ds, 7 * n));
    CK(B.get(&df, 7 * n));
    CK(B.get(&dw, 7 * n));
    CK(B.get(&din, n));
    CK(cudaMemcpy(ds, states, 7 * n * 8, cudaMemcpyHostToDevice));
    rhs_kernel<<<static_cast<unsigned>((n + 127) / 128), 128>>>(ds, n, spin, M, df, dw, din);
    CK(cudaGetLastError());
    CK(cudaMemcpy(fast, df, 7 * n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ieee, dw, 7 * n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(inside, din, n * 4, cudaMemcpyDeviceToHost));
    return 0;
}

// y[i] = grt::pow_quarter(x[i]) evaluated on the device; host arrays of n.
int grt_selftest_pow_quarter(const double* x, size_t n, double* y) {
    if (n == 0) return 0;
    Bufs<2> B;
    double *dx, *dy;
    CK(B.get(&dx, n));
    CK(B.get(&dy, n));
    CK(cudaMemcpy(dx, x, n * 8, cudaMemcpyHostToDevice));
    pow_quarter_kernel<<<static_cast<unsigned>((n + 255) / 256), 256>>>(dx, n, dy);
    CK(cudaGetLastError());
    CK(cudaMemcpy(y, dy, n * 8, cudaMemcpyDeviceToHost));
    return 0;
}

// rcp_box[i] = rcp_rn_box(x[i]), rcp_cuda[i] = __drcp_rn(x[i]),
// sqrt_box[i] = sqrt_rn_box(|x[i]|), sqrt_cuda[i] = sqrt(|x[i]|); host arrays of n.
int grt_selftest_rn_box(const double* x, size_t n, double* rcp_box, double* rcp_cuda, double* sqrt_box,
                        double* sqrt_cuda) {
    if (n == 0) return 0;
    Bufs<5> B;
    double *dx, *d0, *d1, *d2, *d3;
    CK(B.get(&dx, n));
    CK(B.get(&d0, n));
    CK(B.get(&d1, n));
    CK(B.get(&d2, n));
    CK(B.get(&d3, n));
    CK(cudaMemcpy(dx, x, n * 8, cudaMemcpyHostToDevice));
    rn_box_kernel<<<static_cast<unsigned>((n + 255) / 256), 256>>>(dx, n, d0, d1, d2, d3);
    CK(cudaGetLastError());
    CK(cudaMemcpy(rcp_box, d0, n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(rcp_cuda, d1, n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sqrt_box, d2, n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sqrt_cuda, d3, n * 8, cudaMemcpyDeviceToHost));
    return 0;
}

// states as for grt_selftest_rhs; bf / ref receive ks_rhs_rcp<true> /
// ks_rhs_rcp<false>, inside[i] bit 0 / bit 1 their box flags.
int grt_selftest_rhs_bf(const double* states, size_t n, double spin, double M, double* bf, double* ref,
                        uint32_t* inside) {
    if (n == 0) return 0;
    Bufs<4> B;
    double *ds, *db, *dr;
    uint32_t* din;
    CK(B.get(&ds, 7 * n));
    CK(B.get(&db, 7 * n));
    CK(B.get(&dr, 7 * n));
    CK(B.get(&din, n));
    CK(cudaMemcpy(ds, states, 7 * n * 8, cudaMemcpyHostToDevice));
    rhs_bf_kernel<<<static_cast<unsigned>((n + 127) / 128), 128>>>(ds, n, spin, M, db, dr, din);
    CK(cudaGetLastError());
    CK(cudaMemcpy(bf, db, 7 * n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ref, dr, 7 * n * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(inside, din, n * 4, cudaMemcpyDeviceToHost));
    return 0;
}

}  // extern "C"
