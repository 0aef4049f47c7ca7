// The 2-D port-mode eigenproblem on the device: the lowest eigenpairs of
// the generalised problem K v = lambda M v above the gradient null space.
//
// Reference: Numerical2DModeSolver._solve_te_tm
// (src/magnelio/ports/_modal/numerical_2d.py:454-585): K the 2-D curl-curl
// stiffness and M the diagonal epsilon-mass on the free (non-PEC) edges of
// the port plane; the physical modes are the n_modes lowest eigenvalues
// above threshold (the reference keeps lambda > 1e-3 sigma), eigenvectors
// normalised to v^T M v = 1.  The reference runs ARPACK in shift-invert
// mode on the host; here, in float64 on the GPU:
//   1. A = M^-1/2 K M^-1/2 as a dense symmetric matrix,
//   2. Householder tridiagonalisation A = Q T Q^T (one reflector per column:
//      p = A22 v, w = p - (v.p) v, A22 -= 2 (v w^T + w v^T)),
//   3. the wanted eigenvalues of T by bisection on its Sturm sequence,
//   4. their eigenvectors by inverse iteration on T (LU with partial
//      pivoting; vectors of a cluster orthogonalised against each other),
//   5. back to the plane: v = M^-1/2 Q y.
// The sign of each eigenvector is the caller's (the reference fixes it
// from the plane's coordinates).
#include "fitb_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fitb {

namespace {

constexpr int kT = 256;

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, 148LL * 8)); }

__global__ void k_dense_from_csr(long long n, const long long* rp, const long long* col, const double* val,
                                 const double* m, double* A) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double si = 1.0 / sqrt(m[i]);
        for (long long q = rp[i]; q < rp[i + 1]; ++q) {
            const long long j = col[q];
            A[i * n + j] = si * val[q] * (1.0 / sqrt(m[j]));
        }
    }
}

__device__ double block_sum(double x, double* sh) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += sh[w];
        sh[32] = a;
    }
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

// reflector of column k: x = A[k+1:, k]; v = (x - alpha e1) / |x - alpha e1|,
// alpha = -sign(x0) |x|; d[k] = A[k][k], e[k] = alpha; v into V[k][k+1:]
__global__ void __launch_bounds__(kT) k_hh_reflector(long long n, int k, const double* A, double* V, double* d,
                                                      double* e, int* skip) {
    __shared__ double sh[33];
    const long long m = n - k - 1;
    double s = 0.0;
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        const double x = A[(k + 1 + i) * n + k];
        s += x * x;
    }
    const double nx = sqrt(block_sum(s, sh));
    const double x0 = A[(k + 1) * n + k];
    const double alpha = x0 >= 0.0 ? -nx : nx;
    // |x - alpha e1|^2 = |x|^2 - 2 alpha x0 + alpha^2
    const double nv2 = nx * nx - 2.0 * alpha * x0 + alpha * alpha;
    const bool none = nx == 0.0 || nv2 <= 0.0;
    const double inv = none ? 0.0 : 1.0 / sqrt(nv2);
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        const double x = A[(k + 1 + i) * n + k];
        V[(long long)k * n + k + 1 + i] = none ? 0.0 : (x - (i == 0 ? alpha : 0.0)) * inv;
    }
    if (threadIdx.x == 0) {
        d[k] = A[(long long)k * n + k];
        e[k] = none ? x0 : alpha;
        *skip = none ? 1 : 0;
    }
}

// p = A22 v over rows k+1..n-1: one warp per row
__global__ void k_hh_matvec(long long n, int k, const double* A, const double* V, double* p) {
    const long long m = n - k - 1;
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const double* v = V + (long long)k * n + k + 1;
    for (long long r = w0; r < m; r += nw) {
        const double* row = A + (k + 1 + r) * n + k + 1;
        double a = 0.0;
        for (long long j = lane; j < m; j += 32) a += row[j] * v[j];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) p[r] = a;
    }
}

// w = p - (v.p) v
__global__ void __launch_bounds__(kT) k_hh_w(long long n, int k, const double* V, double* p) {
    __shared__ double sh[33];
    const long long m = n - k - 1;
    const double* v = V + (long long)k * n + k + 1;
    double s = 0.0;
    for (long long i = threadIdx.x; i < m; i += blockDim.x) s += v[i] * p[i];
    const double K = block_sum(s, sh);
    for (long long i = threadIdx.x; i < m; i += blockDim.x) p[i] = p[i] - K * v[i];
}

// A22 -= 2 (v w^T + w v^T)
__global__ void k_hh_update(long long n, int k, const double* V, const double* w, double* A, const int* skip) {
    if (*skip) return;
    const long long m = n - k - 1, mm = m * m;
    const double* v = V + (long long)k * n + k + 1;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < mm; t += (long long)gridDim.x * blockDim.x) {
        const long long i = t / m, j = t % m;
        A[(k + 1 + i) * n + k + 1 + j] -= 2.0 * (v[i] * w[j] + w[i] * v[j]);
    }
}

// number of eigenvalues of T below x (Sturm sequence)
__device__ long long sturm_count(const double* d, const double* e, long long n, double x) {
    long long c = 0;
    double q = d[0] - x;
    if (q < 0.0) ++c;
    for (long long i = 1; i < n; ++i) {
        const double qq = q != 0.0 ? q : 1e-300;
        q = (d[i] - x) - e[i - 1] * e[i - 1] / qq;
        if (q < 0.0) ++c;
    }
    return c;
}

// eigenvalues r0 .. r0 + nm - 1 (ascending) of T by bisection; one thread each
__global__ void k_tri_bisect(const double* d, const double* e, long long n, long long r0, int nm, double lo, double hi,
                             double* lam) {
    const int t = threadIdx.x;
    if (t >= nm) return;
    const long long r = r0 + t;
    double a = lo, b = hi;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (a + b);
        if (mid <= a || mid >= b) break;
        if (sturm_count(d, e, n, mid) > r)
            b = mid;
        else
            a = mid;
    }
    lam[t] = 0.5 * (a + b);
}

// eigenvectors of T for lam[0..nm) by inverse iteration (one thread, in
// order; a vector whose eigenvalue is within rel 1e-6 of an earlier one is
// orthogonalised against it); y: [nm][n]; scratch: 5 n doubles
__global__ void k_tri_vectors(const double* d, const double* e, long long n, int nm, const double* lam, double* y,
                              double* wk) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double *l0 = wk, *u0 = wk + n, *u1 = wk + 2 * n, *u2 = wk + 3 * n;
    int* piv = reinterpret_cast<int*>(wk + 4 * n);
    double scale = 0.0;
    for (long long i = 0; i < n; ++i) scale = fmax(scale, fabs(d[i]) + (i ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0));
    for (int q = 0; q < nm; ++q) {
        const double s = lam[q] + 1e-13 * scale;  // keep T - s I off exact singularity
        // LU of T - s I with partial pivoting: rows hold u0 (diag), u1, u2
        double a = d[0] - s, b = n > 1 ? e[0] : 0.0, c = 0.0;
        for (long long i = 0; i < n - 1; ++i) {
            const double sub = e[i], dn = d[i + 1] - s, up = i + 1 < n - 1 ? e[i + 1] : 0.0;
            if (fabs(sub) > fabs(a)) {  // swap rows i and i+1
                piv[i] = 1;
                const double f = a / sub;
                l0[i] = f;
                u0[i] = sub;
                u1[i] = dn;
                u2[i] = up;
                a = b - f * dn;
                b = c - f * up;
            } else {
                piv[i] = 0;
                const double f = a != 0.0 ? sub / a : 0.0;
                l0[i] = f;
                u0[i] = a;
                u1[i] = b;
                u2[i] = c;
                a = dn - f * b;
                b = up - f * c;
            }
            c = 0.0;
        }
        u0[n - 1] = a != 0.0 ? a : 1e-300;
        u1[n - 1] = 0.0;
        u2[n - 1] = 0.0;
        double* x = y + (long long)q * n;
        for (long long i = 0; i < n; ++i) x[i] = 1.0 / sqrt((double)n) * (1.0 + 0.01 * (double)((i * 7919) % 101) / 101.0);
        for (int it = 0; it < 4; ++it) {
            // forward: apply the row swaps and multipliers
            for (long long i = 0; i < n - 1; ++i) {
                if (piv[i]) {
                    const double t = x[i];
                    x[i] = x[i + 1];
                    x[i + 1] = t;
                }
                x[i + 1] -= l0[i] * x[i];
            }
            // back substitution
            for (long long i = n - 1; i >= 0; --i) {
                double v = x[i];
                if (i + 1 < n) v -= u1[i] * x[i + 1];
                if (i + 2 < n) v -= u2[i] * x[i + 2];
                x[i] = v / (u0[i] != 0.0 ? u0[i] : 1e-300);
            }
            // orthogonalise against the earlier vectors of the cluster
            for (int r = 0; r < q; ++r) {
                if (fabs(lam[r] - lam[q]) > 1e-6 * fmax(fabs(lam[q]), 1e-300)) continue;
                const double* z = y + (long long)r * n;
                double dot = 0.0;
                for (long long i = 0; i < n; ++i) dot += z[i] * x[i];
                for (long long i = 0; i < n; ++i) x[i] -= dot * z[i];
            }
            double nn = 0.0;
            for (long long i = 0; i < n; ++i) nn += x[i] * x[i];
            nn = 1.0 / sqrt(nn);
            for (long long i = 0; i < n; ++i) x[i] *= nn;
        }
    }
}

// y <- Q y (reflectors in reverse order), then v = M^-1/2 y; one block per vector
__global__ void __launch_bounds__(kT) k_back_transform(long long n, int nm, const double* V, const double* m, double* y) {
    __shared__ double sh[33];
    double* x = y + (long long)blockIdx.x * n;
    for (long long k = n - 3; k >= 0; --k) {
        const double* v = V + k * n;
        double s = 0.0;
        for (long long i = k + 1 + threadIdx.x; i < n; i += blockDim.x) s += v[i] * x[i];
        const double t = 2.0 * block_sum(s, sh);
        for (long long i = k + 1 + threadIdx.x; i < n; i += blockDim.x) x[i] -= t * v[i];
        __syncthreads();
    }
    for (long long i = threadIdx.x; i < n; i += blockDim.x) x[i] = x[i] / sqrt(m[i]);
}

}  // namespace

int mode_eigensolve(long long n, const long long* rp, const long long* col, const double* val, const double* m,
                    int n_modes, double threshold, double* lam_out, double* vec_out, cudaStream_t s) {
    if (n < 3 || n_modes < 1 || n_modes > 64 || n > 16384) return -1;
    double *A = nullptr, *V = nullptr, *p = nullptr, *d = nullptr, *e = nullptr, *lam = nullptr, *y = nullptr,
           *wk = nullptr;
    int* skip = nullptr;
    auto fail = [&](cudaError_t err) {
        cudaFree(A), cudaFree(V), cudaFree(p), cudaFree(d), cudaFree(e), cudaFree(lam), cudaFree(y), cudaFree(wk),
            cudaFree(skip);
        return err == cudaSuccess ? 0 : -2;
    };
    const size_t nn = (size_t)n * n * sizeof(double);
    if (cudaMalloc(&A, nn) || cudaMalloc(&V, nn) || cudaMalloc(&p, n * sizeof(double)) ||
        cudaMalloc(&d, n * sizeof(double)) || cudaMalloc(&e, n * sizeof(double)) ||
        cudaMalloc(&lam, 64 * sizeof(double)) || cudaMalloc(&y, (size_t)n_modes * n * sizeof(double)) ||
        cudaMalloc(&wk, 5 * n * sizeof(double)) || cudaMalloc(&skip, sizeof(int)))
        return fail(cudaErrorMemoryAllocation);
    cudaMemsetAsync(A, 0, nn, s);
    cudaMemsetAsync(V, 0, nn, s);
    cudaMemsetAsync(e, 0, n * sizeof(double), s);
    k_dense_from_csr<<<blocks_for(n), kT, 0, s>>>(n, rp, col, val, m, A);
    for (int k = 0; k < (int)n - 2; ++k) {
        k_hh_reflector<<<1, kT, 0, s>>>(n, k, A, V, d, e, skip);
        const long long rows = n - k - 1;
        k_hh_matvec<<<blocks_for(rows * 32), kT, 0, s>>>(n, k, A, V, p);
        k_hh_w<<<1, kT, 0, s>>>(n, k, V, p);
        k_hh_update<<<blocks_for(rows * rows), kT, 0, s>>>(n, k, V, p, A, skip);
    }
    // the last 2 x 2 block
    std::vector<double> tail(3);
    cudaMemcpyAsync(&tail[0], A + (n - 2) * n + (n - 2), sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&tail[1], A + (n - 1) * n + (n - 1), sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&tail[2], A + (n - 1) * n + (n - 2), sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(cudaErrorUnknown);
    cudaMemcpyAsync(d + n - 2, &tail[0], sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d + n - 1, &tail[1], sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(e + n - 2, &tail[2], sizeof(double), cudaMemcpyHostToDevice, s);
    // Gerschgorin interval and the index of the first eigenvalue above threshold
    std::vector<double> hd((size_t)n), he((size_t)n);
    cudaMemcpyAsync(hd.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(he.data(), e, n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(cudaErrorUnknown);
    double lo = 1e300, hi = -1e300;
    for (long long i = 0; i < n; ++i) {
        const double r = (i ? std::fabs(he[i - 1]) : 0.0) + (i < n - 1 ? std::fabs(he[i]) : 0.0);
        lo = std::min(lo, hd[i] - r);
        hi = std::max(hi, hd[i] + r);
    }
    auto count = [&](double x) {
        long long c = 0;
        double q = hd[0] - x;
        if (q < 0.0) ++c;
        for (long long i = 1; i < n; ++i) {
            q = (hd[i] - x) - he[i - 1] * he[i - 1] / (q != 0.0 ? q : 1e-300);
            if (q < 0.0) ++c;
        }
        return c;
    };
    const long long r0 = count(threshold);
    if (r0 + n_modes > n) return fail(cudaSuccess) - 3;
    k_tri_bisect<<<1, 64, 0, s>>>(d, e, n, r0, n_modes, std::max(lo, threshold), hi, lam);
    k_tri_vectors<<<1, 32, 0, s>>>(d, e, n, n_modes, lam, y, wk);
    k_back_transform<<<n_modes, kT, 0, s>>>(n, n_modes, V, m, y);
    cudaMemcpyAsync(lam_out, lam, n_modes * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(vec_out, y, (size_t)n_modes * n * sizeof(double), cudaMemcpyDeviceToHost, s);
    const cudaError_t err = cudaStreamSynchronize(s);
    const cudaError_t le = cudaGetLastError();
    return fail(err != cudaSuccess ? err : le);
}

}  // namespace fitb
