// The lowest eigenpairs of a large sparse symmetric positive semi-definite
// matrix on the device, by Chebyshev-filtered subspace iteration in float64.
//
// Used for the port-mode problems of large port planes, where a dense
// eigensolve (modes.cu) is out of reach: the TE modes of a hollow guide as
// the face form L = B B^T, B = W^1/2 C M^-1/2 (C the face circulations of
// the plane's free edges, W = 1/M_mu of the normal-H faces, M the edge
// epsilon-masses), whose nonzero spectrum is that of the edge problem
// K v = lambda M v the reference solves with shift-invert ARPACK
// (src/magnelio/ports/_modal/numerical_2d.py:497-544) and whose null space
// is one known vector per connected face region; and the TM problem on the
// plane's normal edges (curl_curl_2d.py:127-218), positive definite.
//
// One iteration: the block X (n x k, k > n_modes) is passed through the
// Chebyshev polynomial of degree m <= 100 that is bounded by 1 on [a, b]
// (b an upper bound of the spectrum, a the largest Ritz value of the
// block) and grows fast below a (the scaled three-term recurrence, one
// fused SpMM per degree; m capped so that the gain at the lowest Ritz
// value stays near 1e8); the caller's null vectors are projected out; the block is
// orthonormalised by classical Gram-Schmidt with reorthogonalisation; the
// Rayleigh-Ritz step (H = X^T L X, a k x k Jacobi eigensolve on the host)
// rotates it onto the Ritz vectors; the residuals ||L x_j - theta_j x_j||
// decide convergence.  Every loop is bounded; the routine reports the
// iterations used and fails if the residuals do not reach the tolerance.
#include "fitb_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fitb {

namespace {

constexpr int kT = 256;

int grid_for(long long work) {
    return (int)std::max<long long>(1, std::min<long long>((work + kT - 1) / kT, 148LL * 16));
}

// Yn = alpha (L Y) + beta Y + gamma X, blocks column-major (column j at j n)
__global__ void k_cheb(long long n, int k, const long long* rp, const long long* col, const double* val,
                       const double* Y, const double* X, double* Yn, double alpha, double beta, double gamma) {
    const long long total = n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / n, i = t - j * n;
        const double* y = Y + j * n;
        double acc = 0.0;
        for (long long q = rp[i]; q < rp[i + 1]; ++q) acc += val[q] * y[col[q]];
        double r = alpha * acc + beta * y[i];
        if (gamma != 0.0) r += gamma * X[t];
        Yn[t] = r;
    }
}

__device__ double block_reduce(double x, double* sh) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
    return r;
}

// out[i * nb + j] = A_i . B_j for i < na, j < nb (one block per pair)
__global__ void __launch_bounds__(kT) k_gram(long long n, const double* A, int na, const double* B, int nb,
                                             double* out) {
    __shared__ double sh[32];
    const int i = blockIdx.x / nb, j = blockIdx.x - (blockIdx.x / nb) * nb;
    if (i >= na) return;
    const double* a = A + (long long)i * n;
    const double* b = B + (long long)j * n;
    double s = 0.0;
    for (long long r = threadIdx.x; r < n; r += blockDim.x) s += a[r] * b[r];
    s = block_reduce(s, sh);
    if (threadIdx.x == 0) out[i * nb + j] = s;
}

// x_c -= sum_i coef[i * ld + c] A_i for the columns c < nc of X (A has na columns)
__global__ void k_subtract(long long n, double* X, int nc, const double* A, int na, const double* coef, int ld) {
    const long long total = n * nc;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long c = t / n, r = t - c * n;
        double s = 0.0;
        for (int i = 0; i < na; ++i) s += coef[i * ld + c] * A[(long long)i * n + r];
        X[t] -= s;
    }
}

__global__ void k_scale(long long n, double* x, double f) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        x[t] *= f;
}

// Out_j = sum_i In_i R[i * k + j]
__global__ void k_rotate(long long n, int k, const double* In, const double* R, double* Out) {
    const long long total = n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long j = t / n, r = t - j * n;
        double s = 0.0;
        for (int i = 0; i < k; ++i) s += In[(long long)i * n + r] * R[i * k + j];
        Out[t] = s;
    }
}

// out[j] = || W_j - theta_j X_j ||^2 (one block per column)
__global__ void __launch_bounds__(kT) k_residual(long long n, const double* W, const double* X, const double* theta,
                                                 double* out) {
    __shared__ double sh[32];
    const long long j = blockIdx.x;
    const double th = theta[j];
    double s = 0.0;
    for (long long r = threadIdx.x; r < n; r += blockDim.x) {
        const double d = W[j * n + r] - th * X[j * n + r];
        s += d * d;
    }
    s = block_reduce(s, sh);
    if (threadIdx.x == 0) out[j] = s;
}

// a reproducible start block: a hash of (row, column, seed) in [-1, 1)
__global__ void k_random(long long n, int c0, int nc, unsigned seed, double* X) {
    const long long total = n * nc;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long c = t / n + c0, r = t - (t / n) * n;
        unsigned long long h = (unsigned long long)r * 0x9E3779B97F4A7C15ull ^
                               ((unsigned long long)(c + 1) * 0xBF58476D1CE4E5B9ull) ^ ((unsigned long long)seed << 32);
        h ^= h >> 31;
        h *= 0x94D049BB133111EBull;
        h ^= h >> 29;
        X[c * n + r] = (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
}

// symmetric k x k eigen-decomposition by cyclic Jacobi sweeps (bounded):
// values ascending, vectors as the columns of V (row-major k x k)
void jacobi_eigen(int k, std::vector<double> A, std::vector<double>& w, std::vector<double>& V) {
    V.assign((size_t)k * k, 0.0);
    for (int i = 0; i < k; ++i) V[i * k + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < k; ++i) {
            diag += A[i * k + i] * A[i * k + i];
            for (int j = i + 1; j < k; ++j) off += A[i * k + j] * A[i * k + j];
        }
        if (off <= 1e-34 * diag || off == 0.0) break;
        for (int p = 0; p < k; ++p)
            for (int q = p + 1; q < k; ++q) {
                const double apq = A[p * k + q];
                if (apq == 0.0) continue;
                const double theta = (A[q * k + q] - A[p * k + p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int r = 0; r < k; ++r) {
                    const double arp = A[r * k + p], arq = A[r * k + q];
                    A[r * k + p] = c * arp - s * arq;
                    A[r * k + q] = s * arp + c * arq;
                }
                for (int r = 0; r < k; ++r) {
                    const double apr = A[p * k + r], aqr = A[q * k + r];
                    A[p * k + r] = c * apr - s * aqr;
                    A[q * k + r] = s * apr + c * aqr;
                }
                for (int r = 0; r < k; ++r) {
                    const double vrp = V[r * k + p], vrq = V[r * k + q];
                    V[r * k + p] = c * vrp - s * vrq;
                    V[r * k + q] = s * vrp + c * vrq;
                }
            }
    }
    std::vector<int> ord(k);
    for (int i = 0; i < k; ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return A[a * k + a] < A[b * k + b]; });
    std::vector<double> Vs((size_t)k * k);
    w.resize(k);
    for (int j = 0; j < k; ++j) {
        w[j] = A[ord[j] * k + ord[j]];
        for (int r = 0; r < k; ++r) Vs[r * k + j] = V[r * k + ord[j]];
    }
    V.swap(Vs);
}

}  // namespace

int sparse_lowest_eigs(long long n, const long long* rp, const long long* col, const double* val, int n_null,
                       const double* Z, int n_modes, double tol, double b, double* lam_out, double* vec_out,
                       double* res_out, int* iters_out, cudaStream_t s) {
    if (n < 2 || n_modes < 1 || n_modes > 16 || n_null < 0 || n_null > 8) return -1;
    const int k = (int)std::min<long long>(n_modes + std::max(4, n_modes), n - n_null);
    if (k < n_modes || !(b > 0.0)) return -1;
    const size_t blk = (size_t)n * k;
    double *X = nullptr, *Y = nullptr, *Yn = nullptr, *W = nullptr, *sm = nullptr;
    auto release = [&]() { cudaFree(X), cudaFree(Y), cudaFree(Yn), cudaFree(W), cudaFree(sm); };
    if (cudaMalloc(&X, blk * 8) || cudaMalloc(&Y, blk * 8) || cudaMalloc(&Yn, blk * 8) || cudaMalloc(&W, blk * 8) ||
        cudaMalloc(&sm, 4096 * 8)) {
        release();
        return -2;
    }
    double* coef = sm;          // up to 64 coefficients
    double* H = sm + 64;        // k x k
    double* R = sm + 64 + 1024; // k x k
    double* th = sm + 64 + 2048;
    double* rs = sm + 64 + 2048 + 64;
    const int g_blk = grid_for((long long)blk), g_n = grid_for(n);
    auto host_read = [&](const double* d, double* h, int cnt) {
        cudaMemcpyAsync(h, d, cnt * sizeof(double), cudaMemcpyDeviceToHost, s);
        return cudaStreamSynchronize(s) == cudaSuccess;
    };
    // column c of X orthonormal to the null vectors and to columns < c
    auto ortho_column = [&](int c) -> int {
        double* xc = X + (size_t)c * n;
        double before = 0.0, after = 0.0;
        for (int attempt = 0; attempt < 4; ++attempt) {
            k_gram<<<1, kT, 0, s>>>(n, xc, 1, xc, 1, coef);
            if (!host_read(coef, &before, 1)) return -2;
            for (int pass = 0; pass < 2; ++pass) {
                if (n_null) {
                    k_gram<<<n_null, kT, 0, s>>>(n, Z, n_null, xc, 1, coef);
                    k_subtract<<<g_n, kT, 0, s>>>(n, xc, 1, Z, n_null, coef, 1);
                }
                if (c) {
                    k_gram<<<c, kT, 0, s>>>(n, X, c, xc, 1, coef);
                    k_subtract<<<g_n, kT, 0, s>>>(n, xc, 1, X, c, coef, 1);
                }
            }
            k_gram<<<1, kT, 0, s>>>(n, xc, 1, xc, 1, coef);
            if (!host_read(coef, &after, 1)) return -2;
            if (after > 1e-20 * before && after > 0.0) {
                k_scale<<<g_n, kT, 0, s>>>(n, xc, 1.0 / std::sqrt(after));
                return 0;
            }
            // the column lost its rank: start it afresh
            k_random<<<g_n, kT, 0, s>>>(n, c, 1, 7919u * (attempt + 1) + 13u, X);
        }
        return -5;
    };
    std::vector<double> hH((size_t)k * k), w, V, hres(k);
    double a = 0.0, a0 = 0.0, best = 1e300;
    int since_best = 0, it = 0, rc = -4;
    auto rayleigh_ritz = [&]() -> int {
        k_cheb<<<g_blk, kT, 0, s>>>(n, k, rp, col, val, X, X, W, 1.0, 0.0, 0.0);
        k_gram<<<k * k, kT, 0, s>>>(n, X, k, W, k, H);
        if (!host_read(H, hH.data(), k * k)) return -2;
        for (int i = 0; i < k; ++i)
            for (int j = i + 1; j < k; ++j) hH[i * k + j] = hH[j * k + i] = 0.5 * (hH[i * k + j] + hH[j * k + i]);
        jacobi_eigen(k, hH, w, V);
        cudaMemcpyAsync(R, V.data(), (size_t)k * k * sizeof(double), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(th, w.data(), k * sizeof(double), cudaMemcpyHostToDevice, s);
        k_rotate<<<g_blk, kT, 0, s>>>(n, k, X, R, Y);
        k_rotate<<<g_blk, kT, 0, s>>>(n, k, W, R, Yn);
        std::swap(X, Y);
        std::swap(W, Yn);
        k_residual<<<k, kT, 0, s>>>(n, W, X, th, rs);
        if (!host_read(rs, hres.data(), k)) return -2;
        return 0;
    };
    k_random<<<g_blk, kT, 0, s>>>(n, 0, k, 1u, X);
    for (int c = 0; c < k; ++c)
        if (int e = ortho_column(c)) {
            release();
            return e;
        }
    if (int e = rayleigh_ritz()) {
        release();
        return e;
    }
    const int degree = 100, max_iter = 400;
    for (it = 1; it <= max_iter; ++it) {
        a = w[k - 1];
        a0 = std::min(w[0], 0.5 * a);
        if (!(a < b)) a = 0.5 * b;
        // Chebyshev filter of degree `degree` on [a, b], scaled to 1 at a0
        const double e = 0.5 * (b - a), c = 0.5 * (b + a);
        double sigma = e / (a0 - c);
        const double tau = 2.0 / sigma;
        // degree: at most `degree`, and low enough that the filter's gain at
        // the lowest Ritz value over its bound on [a, b] stays near 1e8 (a
        // higher gain would fold the whole block onto one vector)
        const double x0 = (a + b - 2.0 * a0) / (b - a);
        const int m = (int)std::min<double>(degree, std::max(1.0, 19.0 / std::acosh(std::max(x0, 1.0 + 1e-12))));
        k_cheb<<<g_blk, kT, 0, s>>>(n, k, rp, col, val, X, X, Y, sigma / e, -c * sigma / e, 0.0);
        for (int d = 2; d <= m; ++d) {
            const double s2 = 1.0 / (tau - sigma);
            k_cheb<<<g_blk, kT, 0, s>>>(n, k, rp, col, val, Y, X, Yn, 2.0 * s2 / e, -2.0 * s2 * c / e, -sigma * s2);
            std::swap(X, Y);   // X <- Y (previous), Y <- Yn (current)
            std::swap(Y, Yn);
            sigma = s2;
        }
        std::swap(X, Y);       // the filtered block
        for (int cc = 0; cc < k; ++cc)
            if (int er = ortho_column(cc)) {
                release();
                return er;
            }
        if (int er = rayleigh_ritz()) {
            release();
            return er;
        }
        double worst = 0.0;
        for (int j = 0; j < n_modes; ++j) worst = std::max(worst, std::sqrt(std::max(hres[j], 0.0)) / b);
        if (worst <= tol) {
            rc = 0;
            break;
        }
        // residuals stuck at the rounding floor: accept once below 1e-12 b
        if (worst < 0.5 * best) {
            best = worst;
            since_best = 0;
        } else if (++since_best >= 20 && worst <= 1e-12) {
            rc = 0;
            break;
        }
    }
    double worst = 0.0;
    for (int j = 0; j < n_modes; ++j) worst = std::max(worst, std::sqrt(std::max(hres[j], 0.0)) / b);
    if (res_out) *res_out = worst;
    if (iters_out) *iters_out = it;
    if (rc == 0) {
        for (int j = 0; j < n_modes; ++j) lam_out[j] = w[j];
        cudaMemcpyAsync(vec_out, X, (size_t)n_modes * n * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = -2;
    }
    if (cudaGetLastError() != cudaSuccess) rc = -2;
    release();
    return rc;
}

}  // namespace fitb
