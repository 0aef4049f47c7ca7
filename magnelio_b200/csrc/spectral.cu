// Spectral time-step limit on the device: the largest eigenvalue of the
// leapfrog update operator, measured by a Lanczos iteration in float64.
//
// Reference: spectral_dt / _measure_lambda_max
// (src/magnelio/solver/stability.py:296-446): dt = safety * 2 /
// sqrt(lambda_max), lambda_max of the symmetrised operator
// D^-1/2 C^T M_mu^-1 C D^-1/2 (D = M_eps) restricted to the live E edges
// (neither PEC nor M_eps = 0), frozen H faces entering through 1 / M_mu = 0.
// The reference runs ARPACK (Lanczos with implicit restarts) over scipy
// sparse matrices on the host; here the operator is applied matrix-free with
// the engine's padded layout: the curl C of an H face and the dual curl C^T
// of an E edge are the 4-term stencils of the H and E updates, an edge is
// live where its update has beta_E != 0, and the padding entries (zero
// coefficients) drop out.  The Lanczos recursion keeps three vectors; the
// largest eigenvalue of its tridiagonal matrix is found by bisection on the
// Sturm sequence every few steps until it moves by less than `tol`
// (relative).  The extreme Ritz value of plain Lanczos converges without
// reorthogonalisation (lost orthogonality only repeats converged values).
#include "fitb_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fitb {

namespace {

constexpr int kThreads = 256;

template <typename T>
struct OpArgs {
    Geom g;
    const T* meps;  // [3][vol]
    const T* mmu;   // [3][vol]
    const T* bE;    // [3][vol] liveness of E edges
};

template <typename T>
__device__ __forceinline__ double isd(const OpArgs<T>& a, long long o) {
    // D^-1/2 on live edges, 0 elsewhere
    const double m = (double)a.meps[o];
    return (a.bE[o] != T(0) && m > 0.0) ? 1.0 / sqrt(m) : 0.0;
}

// h = M_mu^-1 C (D^-1/2 x) over the padded H box (x in the padded E layout)
template <typename T>
__global__ void k_curl(OpArgs<T> a, const double* __restrict__ x, double* __restrict__ h) {
    const Geom& g = a.g;
    const long long vol = g.vol, si = g.si, sj = g.sj;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < vol; o += (long long)gridDim.x * blockDim.x) {
        // the last plane / row / column have no +1 neighbour in the box
        if (o + si >= vol) {
            h[o] = h[vol + o] = h[2 * vol + o] = 0.0;
            continue;
        }
        auto ev = [&](int c, long long q) { return x[c * vol + q] * isd(a, c * vol + q); };
        const double ex = ev(0, o), ey = ev(1, o), ez = ev(2, o);
        const double cx = ((ev(2, o + sj) - ez) - ev(1, o + 1)) + ey;
        const double cy = ((ev(0, o + 1) - ex) - ev(2, o + si)) + ez;
        const double cz = ((ev(1, o + si) - ey) - ev(0, o + sj)) + ex;
        for (int c = 0; c < 3; ++c) {
            const double m = (double)a.mmu[c * vol + o];
            const double inv = m > 0.0 ? 1.0 / m : 0.0;
            h[c * vol + o] = inv * (c == 0 ? cx : (c == 1 ? cy : cz));
        }
    }
}

// w = D^-1/2 C^T h on live edges; partial sums of w . q per block
template <typename T>
__global__ void k_dual_curl(OpArgs<T> a, const double* __restrict__ h, const double* __restrict__ q,
                            double* __restrict__ w, double* __restrict__ part) {
    const Geom& g = a.g;
    const long long vol = g.vol, si = g.si, sj = g.sj;
    double acc = 0.0;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < vol; o += (long long)gridDim.x * blockDim.x) {
        if (o < si) {  // the first plane has no -1 neighbour in the box (a guard plane: no live edges)
            w[o] = w[vol + o] = w[2 * vol + o] = 0.0;
            continue;
        }
        const double hx = h[o], hy = h[vol + o], hz = h[2 * vol + o];
        const double cx = ((hz - h[2 * vol + o - sj]) - hy) + h[vol + o - 1];
        const double cy = ((hx - h[o - 1]) - hz) + h[2 * vol + o - si];
        const double cz = ((hy - h[vol + o - si]) - hx) + h[o - sj];
        for (int c = 0; c < 3; ++c) {
            const long long e = c * vol + o;
            const double v = isd(a, e) * (c == 0 ? cx : (c == 1 ? cy : cz));
            w[e] = v;
            acc += v * q[e];
        }
    }
    __shared__ double red[kThreads];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// w -= alpha q + beta q_prev; partial sums of |w|^2
__global__ void k_orth(long long n, double alpha, double beta, const double* __restrict__ q,
                       const double* __restrict__ qp, double* __restrict__ w, double* __restrict__ part) {
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double v = w[t] - alpha * q[t] - beta * qp[t];
        w[t] = v;
        acc += v * v;
    }
    __shared__ double red[kThreads];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// q_prev = q; q = w / beta
__global__ void k_shift(long long n, double inv_beta, double* __restrict__ qp, double* __restrict__ q,
                        const double* __restrict__ w) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        qp[t] = q[t];
        q[t] = w[t] * inv_beta;
    }
}

// deterministic start vector on the live edges (a hash of the index); partial |q|^2
template <typename T>
__global__ void k_start(OpArgs<T> a, double* __restrict__ q, double* __restrict__ part) {
    const long long n = 3 * a.g.vol;
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)t * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        const double v = isd(a, t) > 0.0 ? u : 0.0;
        q[t] = v;
        acc += v * v;
    }
    __shared__ double red[kThreads];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_scale(long long n, double s, double* __restrict__ q) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        q[t] *= s;
}

// largest eigenvalue of the symmetric tridiagonal (a, b) by bisection on the
// Sturm sequence count
double tridiag_max(const std::vector<double>& al, const std::vector<double>& be) {
    const int m = (int)al.size();
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < m; ++i) {  // Gershgorin interval
        const double r = (i > 0 ? std::fabs(be[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(be[i]) : 0.0);
        lo = std::min(lo, al[i] - r);
        hi = std::max(hi, al[i] + r);
    }
    auto count_above = [&](double x) {  // eigenvalues > x
        int neg = 0;
        double d = 1.0;
        for (int i = 0; i < m; ++i) {
            const double b2 = i > 0 ? be[i - 1] * be[i - 1] : 0.0;
            d = (al[i] - x) - (i > 0 ? b2 / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0.0) ++neg;
        }
        return m - neg;
    };
    for (int it = 0; it < 200 && hi - lo > 1e-15 * std::fabs(hi); ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count_above(mid) >= 1)
            lo = mid;
        else
            hi = mid;
    }
    return 0.5 * (lo + hi);
}

}  // namespace

template <typename T>
int spectral_lambda(const Geom& g, const T* meps, const T* mmu, const T* bE, int max_iter, double tol, double* lambda,
                    int* iters, cudaStream_t s) {
    const long long n = 3 * g.vol;
    const int blocks = (int)std::min<long long>((g.vol + kThreads - 1) / kThreads, 148LL * 16);
    double *q = nullptr, *qp = nullptr, *w = nullptr, *h = nullptr, *part = nullptr;
    auto cleanup = [&]() {
        for (double* p : {q, qp, w, h, part})
            if (p) cudaFree(p);
    };
    if (cudaMalloc(&q, n * sizeof(double)) != cudaSuccess || cudaMalloc(&qp, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&w, n * sizeof(double)) != cudaSuccess || cudaMalloc(&h, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&part, blocks * sizeof(double)) != cudaSuccess) {
        cleanup();
        return -1;
    }
    std::vector<double> hp(blocks);
    auto sum_parts = [&]() {
        cudaMemcpyAsync(hp.data(), part, blocks * sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        double t = 0.0;
        for (double v : hp) t += v;
        return t;
    };
    OpArgs<T> a{g, meps, mmu, bE};
    cudaMemsetAsync(qp, 0, n * sizeof(double), s);
    k_start<T><<<blocks, kThreads, 0, s>>>(a, q, part);
    const double nq = std::sqrt(sum_parts());
    if (!(nq > 0.0)) {  // no live edge
        cleanup();
        *lambda = 0.0;
        *iters = 0;
        return 0;
    }
    k_scale<<<blocks, kThreads, 0, s>>>(n, 1.0 / nq, q);
    std::vector<double> al, be;
    double beta = 0.0, last = 0.0;
    int it = 0;
    for (; it < max_iter; ++it) {
        k_curl<T><<<blocks, kThreads, 0, s>>>(a, q, h);
        k_dual_curl<T><<<blocks, kThreads, 0, s>>>(a, h, q, w, part);
        const double alpha = sum_parts();
        k_orth<<<blocks, kThreads, 0, s>>>(n, alpha, beta, q, qp, w, part);
        const double b2 = sum_parts();
        al.push_back(alpha);
        beta = std::sqrt(std::max(b2, 0.0));
        if ((it + 1) % 10 == 0 || beta == 0.0) {
            const double cur = tridiag_max(al, be);
            if (it > 20 && std::fabs(cur - last) <= tol * std::fabs(cur)) {
                last = cur;
                ++it;
                break;
            }
            last = cur;
        }
        if (beta == 0.0) {  // invariant subspace: exact
            ++it;
            break;
        }
        be.push_back(beta);
        k_shift<<<blocks, kThreads, 0, s>>>(n, 1.0 / beta, qp, q, w);
    }
    if (be.size() >= al.size()) be.resize(al.size() - 1);
    *lambda = tridiag_max(al, be);
    *iters = it;
    const cudaError_t e = cudaGetLastError();
    cleanup();
    return e == cudaSuccess ? 0 : -2;
}
template int spectral_lambda<float>(const Geom&, const float*, const float*, const float*, int, double, double*, int*,
                                    cudaStream_t);
template int spectral_lambda<double>(const Geom&, const double*, const double*, const double*, int, double, double*,
                                     int*, cudaStream_t);

}  // namespace fitb
