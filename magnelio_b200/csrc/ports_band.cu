// Band-subspace DTBC ports on the device, run with the other port updates
// between the E and the H update.
//
// Reference: PortOperatorBandDTBC.update_e
// (src/magnelio/ports/_modal/band_dtbc.py:1204-1236) over
// BandDTBCBoundary.advance (:618-668), and the recorder's project_V /
// project_I (:1152-1201, recorder.py:236-250).  Per step n of a port and a
// field set, with the boundary state xt (p coordinates):
//   coup    = M_coup x1_prev                    (interior trace, one step old)
//   conv_w  = sum_{j<n} L^out_{n-j} (xt - xt_inc)^j,  xt_inc = sum_{j<n} L^in_{n-j} s^j
//   ghost   = s^n + conv_w;  history^n = (xt - xt_inc, s^n)
//   xt'     = 2 xt - xt_prev - (coup + D0 xt + Dm1 ghost)
//   e[plane] = W xt';  x1_prev = e[x1]
// with the kernel table of the smallest length n0 2^t >= n + 1 (the
// boundary doubles its kernel when a step outgrows it, :591-603).  The
// history sums are split over chunks of kConvChunk steps (k_band_conv) and
// added in chunk order by k_band_port, so the result does not depend on
// scheduling.  All port arithmetic is float64.
#include "fitb_common.cuh"

namespace fitb {

namespace {

constexpr int kBandThreads = 256;
constexpr int kPairs = kBandPMax * kBandPMax / kBandThreads;  // (i, k) pairs per thread

__device__ __forceinline__ long long band_table(const BandDev& d, long long n, long long& len) {
    long long off = 0, L = d.n0;
    while (L < n + 1) {
        off += L;
        L *= 2;
    }
    len = L;
    return off * (long long)d.p * d.p;
}

// chunk c of the history of port blockIdx.z, field set blockIdx.y: partial
// sums of the outgoing and (with an incoming kernel) the incoming terms
__global__ void __launch_bounds__(kBandThreads) k_band_conv(PortsArgs pa, const BandDev* __restrict__ ports) {
    const BandDev& d = ports[blockIdx.z];
    const int b = blockIdx.y, c = blockIdx.x;
    const long long n = *pa.step;
    const long long lo = (long long)c * kConvChunk;
    if (c >= d.conv_chunks || lo >= n) return;
    const long long hi = min(lo + kConvChunk, n);
    const int p = d.p, pp = p * p;
    long long len;
    const long long toff = band_table(d, n, len);
    __shared__ double red[kBandPMax * kBandPMax];
    for (int dir = 0; dir < (d.has_in ? 2 : 1); ++dir) {
        const double* L = (dir == 0 ? d.kout : d.kin) + toff;
        const double* hist = (dir == 0 ? d.whist : d.shist) + (long long)b * d.cap * p;
        double acc[kPairs];
#pragma unroll
        for (int q = 0; q < kPairs; ++q) acc[q] = 0.0;
        for (long long j = lo; j < hi; ++j) {
            const double* Lm = L + (n - j) * pp;
            const double* w = hist + j * p;
#pragma unroll
            for (int q = 0; q < kPairs; ++q) {
                const int t = threadIdx.x + q * kBandThreads;
                if (t < pp) acc[q] += Lm[t] * w[t % p];
            }
        }
#pragma unroll
        for (int q = 0; q < kPairs; ++q) {
            const int t = threadIdx.x + q * kBandThreads;
            if (t < pp) red[t] = acc[q];
        }
        __syncthreads();
        if (threadIdx.x < p) {
            double a = 0.0;
            for (int k = 0; k < p; ++k) a += red[threadIdx.x * p + k];
            d.conv[(((long long)b * d.conv_chunks + c) * 2 + dir) * p + threadIdx.x] = a;
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kBandThreads)
    k_band_port(T* __restrict__ e, const T* __restrict__ h, PortsArgs pa, const BandDev* __restrict__ ports) {
    const BandDev& d = ports[blockIdx.x];
    const int b = blockIdx.y;
    const long long n = *pa.step;
    const int p = d.p, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kBandThreads / 32;
    T* E = e + (long long)b * pa.e_block;
    const T* H = h + (long long)b * pa.h_block;
    double* st = d.st + (long long)b * 2 * p;
    double* x1p = d.x1prev + (long long)b * d.n1;
    __shared__ double xt[kBandPMax], xtp[kBandPMax], coup[kBandPMax], ghost[kBandPMax], xtn[kBandPMax];
    __shared__ double wred[NW][2 * kMaxModes];
    if (tid < p) {
        xt[tid] = st[tid];
        xtp[tid] = st[p + tid];
    }
    // coup = M_coup x1_prev: one warp per row, lanes over the trace
    for (int i = warp; i < p; i += NW) {
        double a = 0.0;
        for (long long q = lane; q < d.n1; q += 32) a += d.Mc[(long long)i * d.n1 + q] * x1p[q];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) coup[i] = a;
    }
    __syncthreads();
    if (tid < p) {
        const int i = tid;
        const int nck = (int)((n + kConvChunk - 1) / kConvChunk);
        double cw = 0.0, xi = 0.0;
        for (int c = 0; c < nck; ++c) {
            const double* part = d.conv + (((long long)b * d.conv_chunks + c) * 2) * p;
            cw += part[i];
            if (d.has_in) xi += part[p + i];
        }
        const double s = (d.src_on[b] && n < d.n_src) ? d.src[((long long)b * d.n_src + n) * p + i] : 0.0;
        d.whist[((long long)b * d.cap + n) * p + i] = xt[i] - xi;
        d.shist[((long long)b * d.cap + n) * p + i] = s;
        ghost[i] = s + cw;
    }
    __syncthreads();
    if (tid < p) {
        const int i = tid;
        double a0 = 0.0, am = 0.0;
        for (int k = 0; k < p; ++k) a0 += d.D0[i * p + k] * xt[k];
        for (int k = 0; k < p; ++k) am += d.Dm1[i * p + k] * ghost[k];
        const double v = (2.0 * xt[i] - xtp[i]) - ((coup[i] + a0) + am);
        xtn[i] = v;
        st[i] = v;
        st[p + i] = xt[i];
    }
    __syncthreads();
    // port plane from xt', and the recorder's V from the stored values
    // (u part and v part summed separately, then added, per channel)
    double acc[2 * kMaxModes];
#pragma unroll
    for (int m = 0; m < 2 * kMaxModes; ++m) acc[m] = 0.0;
    const int M = d.M;
    const long long nt = d.n_u + d.n_v;
    for (long long r = tid; r < d.n_u; r += kBandThreads) {
        double v = 0.0;
        for (int k = 0; k < p; ++k) v += d.Wu[r * p + k] * xtn[k];
        const T stored = (T)v;
        E[d.eu[r]] = stored;
        const double ev = (double)stored, me = d.me[r];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[m] += me * (d.vprof[(long long)m * nt + r] * ev);
    }
    for (long long r = tid; r < d.n_v; r += kBandThreads) {
        double v = 0.0;
        for (int k = 0; k < p; ++k) v += d.Wv[r * p + k] * xtn[k];
        const T stored = (T)v;
        E[d.ev[r]] = stored;
        const double ev = (double)stored, me = d.me[d.n_u + r];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[kMaxModes + m] += me * (d.vprof[(long long)m * nt + d.n_u + r] * ev);
    }
    // V: the u and v sums of each channel
#pragma unroll
    for (int q = 0; q < 2 * kMaxModes; ++q) {
        const int m = q % kMaxModes;
        if (m >= M) continue;
        double x = acc[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) wred[warp][q < kMaxModes ? m : M + m] = x;
    }
    __syncthreads();
    __shared__ double sv[2 * kMaxModes];
    if (tid < 2 * M) {
        double a = 0.0;
        for (int w = 0; w < NW; ++w) a += wred[w][tid];
        sv[tid] = a;
    }
    __syncthreads();
    // I from h^{n+1/2} on the dual faces
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) acc[m] = 0.0;
    for (long long q = tid; q < d.n_h; q += kBandThreads) {
        const double hv = (double)H[d.hh[q]], mh = d.mh[q];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[m] += mh * (d.hprof[(long long)m * d.n_h + q] * hv);
    }
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) {
        if (m >= M) continue;
        double x = acc[m];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) wred[warp][m] = x;
    }
    __syncthreads();
    if (tid < M) {
        const int m = tid;
        double a = 0.0;
        for (int w = 0; w < NW; ++w) a += wred[w][m];
        const double V = (sv[m] + sv[M + m]) * d.rec_scale[m], I = a * d.rec_scale[m];
        const long long r = ((long long)b * pa.rec.cap + n) * pa.rec.nch + d.channel0 + m;
        pa.rec.V[r] = V;
        pa.rec.I[r] = I;
        // non-negative doubles order like their bit patterns; fmax drops a NaN
        atomicMax(reinterpret_cast<unsigned long long*>(pa.absmax + b),
                  (unsigned long long)__double_as_longlong(fmax(0.0, fabs(V))));
    }
    // the new interior trace: after this port's writes (other entries)
    for (long long q = tid; q < d.n1; q += kBandThreads) x1p[q] = (double)E[d.x1[q]];
}

}  // namespace

template <typename T>
void launch_band(T* e, const T* h, const PortsArgs& pa, const BandDev* d, int n_band, int max_chunks, cudaStream_t s) {
    if (n_band <= 0) return;
    if (max_chunks > 0) k_band_conv<<<dim3(max_chunks, pa.B, n_band), kBandThreads, 0, s>>>(pa, d);
    k_band_port<T><<<dim3(n_band, pa.B), kBandThreads, 0, s>>>(e, h, pa, d);
}
template void launch_band<float>(float*, const float*, const PortsArgs&, const BandDev*, int, int, cudaStream_t);
template void launch_band<double>(double*, const double*, const PortsArgs&, const BandDev*, int, int, cudaStream_t);

}  // namespace fitb
