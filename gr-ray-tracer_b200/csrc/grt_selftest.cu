// Device self-checks of the reciprocal quotients of the FP64 right-hand side,
// built into lib/libgrt_selftest.so (test infrastructure; the product library
// does not link it), with -fmad=false like the trace kernels.
//   grt_selftest_division  div_by(a, b, RN(1/b)) and IEEE a / b on the same operands;
//   grt_selftest_rhs       ks_rhs_rcp (and its box flag) and ks_rhs on the same states;
//   grt_selftest_pow_quarter  the RK45 controller's pow_quarter on the device.
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

}  // extern "C"
