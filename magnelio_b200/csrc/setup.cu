// Per-request setup on the device.
//
// Material matrices and leapfrog coefficients built from the grid and the
// cell materials, for problems whose host would otherwise compute and
// upload six float64 arrays of ~3 entries per cell.  And the DTBC kernel
// tables of the modal ports (below).
//
// Reference: build_M_eps (src/magnelio/_operators/material_matrices.py
// :334-464: cat-0 permittivity of the clamped owner cell times the edge's
// A_dual / L_primal, cat-1 edges overridden with their averaged
// permittivity), build_M_mu (:494-531, non-magnetic: MU0 A_primal /
// L_dual), the lossless leapfrog coefficients alpha = (M - dt sigma / 2) /
// (M + dt sigma / 2), beta = dt / (M + dt sigma / 2) with M = 0 entries
// frozen at (1, 0) (src/magnelio/solver/fit_td.py:383-461), and PEC edges
// frozen at (0, 0) (fit_td.py:497-513).  Every product and quotient is
// rounded as written, in the order the host restatement
// (magnelio_b200/host.py build_M_eps, build_M_mu, leapfrog_coefficients)
// evaluates it, so both give the same bits.
#include "fitb_common.cuh"

#include <algorithm>

namespace fitb {

namespace {

constexpr double kMU0 = 1.25663706212e-6;  // CODATA 2018
constexpr double kC0 = 299792458.0;

// dual width of node n of an axis with cell widths d[0 .. nc-1]: the full end
// cell at the boundary, the mean of the two neighbours inside
__device__ __forceinline__ double dual_w(const double* d, int nc, int n) {
    if (n == 0) return d[0];
    if (n >= nc) return d[nc - 1];
    return __dmul_rn(0.5, __dadd_rn(d[n - 1], d[n]));
}

struct MatArgs {
    Geom g;
    const double *dx, *dy, *dz;
    const int* mat;       // [nx][ny][nz] material of each cell
    const double* eps_r;  // per material
    double eps0, dt;
};

// flat reference index of one E (side 0) or H (side 1) entry -> component and
// (i, j, k)
__device__ __forceinline__ void unflatten(const Geom& g, int side, long long q, int& c, int& i, int& j, int& k) {
    for (c = 0; c < 3; ++c) {
        int ni, nj, nk;
        comp_shape(g, 3 * side + c, ni, nj, nk);
        const long long n = (long long)ni * nj * nk;
        if (q < n) {
            k = (int)(q % nk);
            const long long r = q / nk;
            j = (int)(r % nj);
            i = (int)(r / nj);
            return;
        }
        q -= n;
    }
}

// (M, alpha, beta) of one E edge from its permittivity (relative, times EPS0)
template <typename T>
__device__ __forceinline__ void put_E(const MatArgs& a, T* aE, T* bE, T* meps, int c, int i, int j, int k, double eps) {
    const Geom& g = a.g;
    double geo;
    if (c == 0)
        geo = __ddiv_rn(__dmul_rn(dual_w(a.dy, g.ny, j), dual_w(a.dz, g.nz, k)), a.dx[i]);
    else if (c == 1)
        geo = __ddiv_rn(__dmul_rn(dual_w(a.dx, g.nx, i), dual_w(a.dz, g.nz, k)), a.dy[j]);
    else
        geo = __ddiv_rn(__dmul_rn(dual_w(a.dx, g.nx, i), dual_w(a.dy, g.ny, j)), a.dz[k]);
    const double M = __dmul_rn(__dmul_rn(a.eps0, eps), geo);
    const bool live = M > 0.0;
    const double den = live ? __dadd_rn(M, 0.0) : 1.0;
    const double al = live ? __ddiv_rn(__dsub_rn(M, 0.0), den) : 1.0;
    const double be = live ? __ddiv_rn(a.dt, den) : 0.0;
    const long long o = (long long)c * g.vol + pidx(g, i, j, k);
    aE[o] = (T)al;
    bE[o] = (T)be;
    meps[o] = (T)M;
}

template <typename T>
__global__ void k_setup_E(MatArgs a, long long n_e, T* aE, T* bE, T* meps) {
    const Geom& g = a.g;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_e;
         q += (long long)gridDim.x * blockDim.x) {
        int c, i, j, k;
        unflatten(g, 0, q, c, i, j, k);
        // the owner cell, clamped at the domain boundary
        const int ic = c == 0 ? i : min(i, g.nx - 1), jc = c == 1 ? j : min(j, g.ny - 1),
                  kc = c == 2 ? k : min(k, g.nz - 1);
        const double eps = a.eps_r[a.mat[((long long)ic * g.ny + jc) * g.nz + kc]];
        put_E(a, aE, bE, meps, c, i, j, k, eps);
    }
}

// cat-1 edges: the averaged permittivity replaces the owner cell's
template <typename T>
__global__ void k_setup_cat1(MatArgs a, long long n, const long long* idx, const double* eps, T* aE, T* bE,
                             T* meps) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        int c, i, j, k;
        unflatten(a.g, 0, idx[q], c, i, j, k);
        put_E(a, aE, bE, meps, c, i, j, k, eps[q]);
    }
}

template <typename T>
__global__ void k_setup_pec(Geom g, long long n, const long long* idx, T* aE, T* bE) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        int c, i, j, k;
        unflatten(g, 0, idx[q], c, i, j, k);
        const long long o = (long long)c * g.vol + pidx(g, i, j, k);
        aE[o] = T(0);
        bE[o] = T(0);
    }
}

// non-magnetic M_mu and the H coefficients
template <typename T>
__global__ void k_setup_H(MatArgs a, long long n_h, T* aH, T* bH, T* mmu) {
    const Geom& g = a.g;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_h;
         q += (long long)gridDim.x * blockDim.x) {
        int c, i, j, k;
        unflatten(g, 1, q, c, i, j, k);
        double M;
        if (c == 0)
            M = __ddiv_rn(__dmul_rn(__dmul_rn(kMU0, a.dy[j]), a.dz[k]), dual_w(a.dx, g.nx, i));
        else if (c == 1)
            M = __ddiv_rn(__dmul_rn(__dmul_rn(kMU0, a.dx[i]), a.dz[k]), dual_w(a.dy, g.ny, j));
        else
            M = __ddiv_rn(__dmul_rn(__dmul_rn(kMU0, a.dx[i]), a.dy[j]), dual_w(a.dz, g.nz, k));
        const bool live = M > 0.0;
        const double den = live ? __dadd_rn(M, 0.0) : 1.0;
        const double al = live ? __ddiv_rn(__dsub_rn(M, 0.0), den) : 1.0;
        const double be = live ? __ddiv_rn(a.dt, den) : 0.0;
        const long long o = (long long)c * g.vol + pidx(g, i, j, k);
        aH[o] = (T)al;
        bH[o] = (T)be;
        mmu[o] = (T)M;
    }
}

__device__ __forceinline__ void atomic_max_abs(double* addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(fabs(v)));
}

// per-component max |x| of the four coefficient arrays (out[4][3]) over the
// padded boxes (the padding holds zeros)
template <typename T>
__global__ void k_coef_max(long long vol, const T* aE, const T* bE, const T* aH, const T* bH, double* out) {
    double m[12] = {};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < vol;
         q += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; ++c) {
            const long long o = c * vol + q;
            m[c] = fmax(m[c], fabs((double)aE[o]));
            m[3 + c] = fmax(m[3 + c], fabs((double)bE[o]));
            m[6 + c] = fmax(m[6 + c], fabs((double)aH[o]));
            m[9 + c] = fmax(m[9 + c], fabs((double)bH[o]));
        }
    for (int r = 0; r < 12; ++r) {
        double v = m[r];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) atomic_max_abs(out + r, v);
    }
}

int grid_of(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 32); }

// ---------------------------------------------------------------------------
// DTBC kernel table (dtbc.py:91-156): l_m = rho^m Re(c_m), m < n, where
// c_m = (1/N) sum_k lambda(z_k) e^{2 pi i k m / N} is the inverse DFT of the
// outgoing root on N = 8 n points z_k = rho e^{2 pi i k / N} of the circle
// rho = exp(4 / n).  The reference takes the inverse FFT of the N samples;
// here each coefficient is one direct sum (N terms) in float64.

struct Cx {
    double re, im;
};

__device__ __forceinline__ Cx cx_mul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

// principal square root by the scaled formula of Numerical Recipes (section
// 5.5): t = sqrt((|a| + |w|) / 2), then the quotient for the other part
__device__ __forceinline__ Cx cx_sqrt(Cx w) {
    if (w.re == 0.0 && w.im == 0.0) return {0.0, 0.0};
    const double t = sqrt(0.5 * (fabs(w.re) + hypot(w.re, w.im)));
    if (w.re >= 0.0) return {t, w.im / (2.0 * t)};
    return {fabs(w.im) / (2.0 * t), copysign(t, w.im)};
}

// lambda(z) of dtbc.py:91-122: A = 1 + (z - 2 + 1/z + q^2) / (2 r^2), the
// root of A +- sqrt(A^2 - 1) of modulus <= 1
__global__ void k_dtbc_samples(double r, double q, long long N, double rho, double2* x) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N; k += (long long)gridDim.x * blockDim.x) {
        double sn, cs;
        sincospi(2.0 * (double)k / (double)N, &sn, &cs);
        const Cx z{rho * cs, rho * sn};
        const double zz = z.re * z.re + z.im * z.im;
        const Cx iz{z.re / zz, -z.im / zz};
        const double den = 2.0 * r * r;
        const Cx A{1.0 + (z.re - 2.0 + iz.re + q * q) / den, (z.im + iz.im) / den};
        const Cx A2 = cx_mul(A, A);
        const Cx root = cx_sqrt({A2.re - 1.0, A2.im});
        const Cx lm{A.re - root.re, A.im - root.im}, lp{A.re + root.re, A.im + root.im};
        const Cx lam = hypot(lm.re, lm.im) <= hypot(lp.re, lp.im) ? lm : lp;
        x[k] = make_double2(lam.re, lam.im);
    }
}

// one CTA per coefficient m: thread t sums its contiguous run of k with a
// rotated phasor restarted from sincospi every kRestart terms, then a fixed
// reduction order (warp tree, then warps in order)
constexpr int kDftThreads = 256, kRestart = 32;

__global__ void __launch_bounds__(kDftThreads) k_dtbc_coeffs(const double2* __restrict__ x, long long N, double rho,
                                                              double* __restrict__ l) {
    const int m = blockIdx.x;
    const long long per = (N + kDftThreads - 1) / kDftThreads;
    const long long k0 = threadIdx.x * per, k1 = min(N, k0 + per);
    double sw, cw;
    sincospi(2.0 * (double)(m % N) / (double)N, &sw, &cw);  // e^{2 pi i m / N}
    double acc = 0.0;
    for (long long kb = k0; kb < k1; kb += kRestart) {
        double sn, cs;
        sincospi(2.0 * (double)((kb * (long long)m) % N) / (double)N, &sn, &cs);
        const long long ke = min(k1, kb + kRestart);
        for (long long k = kb; k < ke; ++k) {
            const double2 v = x[k];
            acc += v.x * cs - v.y * sn;  // Re(x_k e^{i theta_k m})
            const double c2 = cs * cw - sn * sw, s2 = sn * cw + cs * sw;
            cs = c2;
            sn = s2;
        }
    }
    __shared__ double ws[kDftThreads / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < kDftThreads / 32; ++w) a += ws[w];
        l[m] = (a * (1.0 / (double)N)) * pow(rho, (double)m);
    }
}

}  // namespace

void launch_dtbc_kernel(double r, double q, int n, double2* x, double* l, cudaStream_t s) {
    const long long N = 8LL * n;
    const double rho = exp(4.0 / (double)n);
    k_dtbc_samples<<<grid_of(N), 256, 0, s>>>(r, q, N, rho, x);
    k_dtbc_coeffs<<<n, kDftThreads, 0, s>>>(x, N, rho, l);
}

template <typename T>
void launch_setup_materials(const Geom& g, const double* dx, const double* dy, const double* dz, const int* mat,
                            const double* eps_r, double dt, long long n_cat1, const long long* cat1_idx,
                            const double* cat1_eps, long long n_pec, const long long* pec_idx, T* aE, T* bE, T* aH,
                            T* bH, T* meps, T* mmu, double* coef_max, cudaStream_t s) {
    MatArgs a{g, dx, dy, dz, mat, eps_r, 1.0 / (kMU0 * kC0 * kC0), dt};
    const long long n_e = (long long)g.nx * (g.ny + 1) * (g.nz + 1) + (long long)(g.nx + 1) * g.ny * (g.nz + 1) +
                          (long long)(g.nx + 1) * (g.ny + 1) * g.nz;
    const long long n_h = (long long)(g.nx + 1) * g.ny * g.nz + (long long)g.nx * (g.ny + 1) * g.nz +
                          (long long)g.nx * g.ny * (g.nz + 1);
    k_setup_E<T><<<grid_of(n_e), 256, 0, s>>>(a, n_e, aE, bE, meps);
    if (n_cat1 > 0) k_setup_cat1<T><<<grid_of(n_cat1), 256, 0, s>>>(a, n_cat1, cat1_idx, cat1_eps, aE, bE, meps);
    if (n_pec > 0) k_setup_pec<T><<<grid_of(n_pec), 256, 0, s>>>(g, n_pec, pec_idx, aE, bE);
    k_setup_H<T><<<grid_of(n_h), 256, 0, s>>>(a, n_h, aH, bH, mmu);
    cudaMemsetAsync(coef_max, 0, 12 * sizeof(double), s);
    k_coef_max<T><<<grid_of(g.vol), 256, 0, s>>>(g.vol, aE, bE, aH, bH, coef_max);
}
template void launch_setup_materials<float>(const Geom&, const double*, const double*, const double*, const int*,
                                            const double*, double, long long, const long long*, const double*,
                                            long long, const long long*, float*, float*, float*, float*, float*,
                                            float*, double*, cudaStream_t);
template void launch_setup_materials<double>(const Geom&, const double*, const double*, const double*, const int*,
                                             const double*, double, long long, const long long*, const double*,
                                             long long, const long long*, double*, double*, double*, double*,
                                             double*, double*, double*, cudaStream_t);

}  // namespace fitb
