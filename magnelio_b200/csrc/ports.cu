// Port terminations on the device, run between the E and H updates.
//
// Lumped ports: LumpedElementOperator.update_e
//   (src/magnelio/ports/_lumped/operator.py:134-166) with the series R-L-C
//   trapezoidal companion (src/magnelio/circuit/companion.py SeriesRLC).
// Modal ports: PortOperatorModal.update_e
//   (src/magnelio/ports/_modal/operator.py:1351-1536): interior-plane
//   projection, modal Mur-1 / TF-SF, the exact DTBC chain step
//   (src/magnelio/ports/_modal/dtbc.py:417-463), modal reconstruction of the
//   port plane, the complement absorber, then the V/I samples the recorder
//   takes right after update_e (src/magnelio/ports/recorder.py:216-252).
// All port arithmetic is float64, as in the reference; only the field
// gathers/scatters touch the field dtype.
#include "fitb_common.cuh"

namespace fitb {

namespace {

constexpr int kPortThreads = 256;

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    // Non-negative doubles order like their bit patterns.
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// Block-wide sums of the per-thread partial sums v[m], m < M, into red[m]
// and, with PAIRS, of v[kMaxModes + m] into red[M + m]; valid in red for all
// threads after return.  The mode loops are unrolled to kMaxModes with a
// guard, so that v stays in registers; each value is summed by the same
// shuffle tree and then in warp order.
template <bool PAIRS>
__device__ void block_sum_modes(const double (&v)[2 * kMaxModes], int M, double* red,
                                double (*wred)[2 * kMaxModes]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < (PAIRS ? 2 : 1) * kMaxModes; ++q) {
        const int m = q % kMaxModes;
        if (m >= M) continue;  // uniform over the block
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) wred[warp][q < kMaxModes ? m : M + m] = x;
    }
    __syncthreads();
    if (threadIdx.x < (PAIRS ? 2 : 1) * M) {
        double acc = 0.0;
        for (int w = 0; w < nwarps; ++w) acc += wred[w][threadIdx.x];
        red[threadIdx.x] = acc;
    }
    __syncthreads();
}

template <typename T>
__global__ void k_lumped(T* __restrict__ e, PortsArgs pa, const LumpedDev* __restrict__ ports) {
    const LumpedDev& d = ports[blockIdx.x];
    const int b = blockIdx.y;
    if (threadIdx.x != 0) return;
    const long long n = *pa.step;
    T* E = e + (long long)b * pa.e_block;
    double v_total = 0.0;
    for (int q = 0; q < d.n_edges; ++q) v_total += d.sign[q] * (double)E[d.off[q]];
    const double v_src = (n < d.n_src) ? d.src[(long long)b * d.n_src + n] : 0.0;
    double* st = d.st + 4 * b;
    const double dt = pa.dt_lumped;
    const double i_prev = st[0];
    double r_eq = (d.R >= 0.0) ? d.R : 0.0;
    if (d.L >= 0.0) r_eq += 2.0 * d.L / dt;
    if (d.C >= 0.0) r_eq += dt / (2.0 * d.C);
    double v_hist = 0.0;
    if (d.L >= 0.0) v_hist += -(2.0 * d.L / dt) * i_prev - st[1];
    if (d.C >= 0.0) v_hist += st[2] + (dt / (2.0 * d.C)) * i_prev;
    const double z_eff = r_eq + d.beta_sum;
    const double i_port = (v_src - v_hist - v_total) / z_eff;
    for (int q = 0; q < d.n_edges; ++q) {
        const long long o = d.off[q];
        E[o] = (T)((double)E[o] + d.sign[q] * d.beta[q] * i_port);
    }
    if (d.L >= 0.0) st[1] = (2.0 * d.L / dt) * (i_port - i_prev) - st[1];
    if (d.C >= 0.0) st[2] = st[2] + (dt / (2.0 * d.C)) * (i_port + i_prev);
    st[0] = i_port;
    st[3] = i_port;
    // Recorder: V re-projected from the corrected field, I = cached current.
    double v = 0.0;
    for (int q = 0; q < d.n_edges; ++q) v += d.sign[q] * (double)E[d.off[q]];
    const long long r = ((long long)b * pa.rec.cap + n) * pa.rec.nch + d.channel;
    pa.rec.V[r] = v * d.rec_scale;
    pa.rec.I[r] = i_port * d.rec_scale;
}

// _interp_delayed (operator.py:1539-1562) on the source history
// wf[0..n+1], whose deque holds the last `maxlen` samples.
__device__ __forceinline__ double interp_delayed(const double* wf, long long n_wf, long long n,
                                                 int maxlen, double delay, double dt) {
    const long long len = min(n + 1, (long long)maxlen);
    const double idx_frac = delay / dt;
    const long long i0 = (long long)floor(idx_frac);
    const double alpha = idx_frac - (double)i0;
    if (len - 1 - i0 < 0) return 0.0;
    const long long t0 = n + 1 - i0;
    const double v0 = (t0 >= 0 && t0 < n_wf) ? wf[t0] : 0.0;
    double v1 = 0.0;
    if (len - 2 - i0 >= 0) {
        const long long t1 = n - i0;
        v1 = (t1 >= 0 && t1 < n_wf) ? wf[t1] : 0.0;
    }
    return (1.0 - alpha) * v0 + alpha * v1;
}

template <typename T>
__global__ void __launch_bounds__(kPortThreads)
    k_modal(T* __restrict__ e, const T* __restrict__ h, PortsArgs pa,
            const ModalDev* __restrict__ ports) {
    // The phases below keep the reference's arithmetic per value; what moves
    // is when the loads happen: everything that does not depend on this
    // step's port update (the mode state, the DTBC partial sums, the H
    // samples of the recorder) is read up front, so that a step costs few
    // dependent memory round trips.
    const ModalDev& d = ports[blockIdx.x];
    const int b = blockIdx.y;
    const long long n = *pa.step;
    const int M = d.n_modes, ne = d.n_e, nh = d.n_h;
    T* E = e + (long long)b * pa.e_block;
    const T* H = h + (long long)b * pa.h_block;
    double* st = d.st + (long long)b * 4 * kMaxModes;
    double* Vport_prev = st;
    double* Vint_prev = st + kMaxModes;
    double* u = st + 2 * kMaxModes;
    double* u_prev = st + 3 * kMaxModes;
    double* eint = d.scratch + (long long)b * 2 * ne;
    double* enew = eint + ne;

    __shared__ double red[2 * kMaxModes];
    __shared__ double wred[kPortThreads / 32][2 * kMaxModes];
    __shared__ double s_vint[kMaxModes];
    __shared__ double s_vc[kMaxModes];
    __shared__ double s_conv[2 * kMaxModes];

    // mode state of mode m = threadIdx.x (m < M)
    const int exc = d.exc_mode[b];
    const int tm = threadIdx.x < M ? threadIdx.x : 0;
    const double vport0 = Vport_prev[tm], vint0 = Vint_prev[tm], u0 = u[tm], up0 = u_prev[tm];
    const double mur = d.mur_r[tm];
    const bool dtbc = d.is_dtbc[tm];
    const double r2 = d.r2[tm], q2 = d.q2[tm];
    // the excitation samples this step needs (they do not depend on the
    // fields): Mur TF/SF source terms, or the DTBC ghost source
    double src_new = 0.0, inc_int_now = 0.0, inc_int_prev = 0.0, inc_face_prev = 0.0, src_dtbc = 0.0;
    if (threadIdx.x < M && tm == exc) {
        const double* wf = d.wf + (long long)b * d.n_wf;
        if (!dtbc) {
            const long long t1 = n + 1;
            src_new = (t1 < d.n_wf) ? wf[t1] : 0.0;
            const int maxlen = d.buf_len[b];
            inc_int_now = interp_delayed(wf, d.n_wf, n, maxlen, d.tau[tm], d.dt);
            inc_int_prev = interp_delayed(wf, d.n_wf, n, maxlen, d.tau[tm] + d.dt, d.dt);
            inc_face_prev = interp_delayed(wf, d.n_wf, n, maxlen, d.dt, d.dt);
        } else {
            src_dtbc = n < d.n_wf ? wf[n] : 0.0;
        }
    }

    // 2. DTBC boundary convolutions conv_w = sum_{m=1..n} l_m w[n-m] and
    //    u_inc = sum l_m s[n-m]: the partial sums k_dtbc_conv left per
    //    history chunk (before this kernel, on the same stream), added in
    //    chunk order (a fixed order: the result does not depend on
    //    scheduling).
    if (threadIdx.x < 2 * M && d.is_dtbc[threadIdx.x >> 1]) {
        const int m = threadIdx.x >> 1, w = threadIdx.x & 1;
        const int nck = (int)((n + kConvChunk - 1) / kConvChunk);
        const double* part = d.conv + (((long long)b * M + m) * d.conv_chunks) * 2 + w;
        double a = 0.0;
        for (int c = 0; c < nck; ++c) a += part[2 * c];
        s_conv[threadIdx.x] = a;
    }

    // 1. Interior-plane projection V_int_new[m] = sum me_int * (p_m * e_int),
    //    and the recorder's I samples from h^{n+1/2} (this kernel writes no
    //    H) into acc[kMaxModes + m].  The mode loops are unrolled to
    //    kMaxModes with a guard so that the partial sums stay in registers.
    double acc[2 * kMaxModes];
#pragma unroll
    for (int m = 0; m < 2 * kMaxModes; ++m) acc[m] = 0.0;
    const bool split = d.n_chunks > 1;
    if (split) {
        // a large plane: k_modal_gather left one partial sum per chunk of
        // edges (and faces); added here in chunk order
        if (threadIdx.x < 2 * M) {
            const double* pp = d.part + (long long)b * d.n_chunks * 2 * kMaxModes + threadIdx.x;
            double a = 0.0;
            for (int c = 0; c < d.n_chunks; ++c) a += pp[(long long)c * 2 * kMaxModes];
            red[threadIdx.x] = a;
        }
        __syncthreads();
    }
    for (int p = split ? ne : threadIdx.x; p < ne; p += blockDim.x) {
        const double v = (double)E[d.int_e[p]];
        eint[p] = v;
        const double me = d.me_int[p];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[m] += me * (d.vprof[(long long)m * ne + p] * v);
    }
    for (int p = split ? nh : threadIdx.x; p < nh; p += blockDim.x) {
        const double v = (double)H[d.port_h[p]];
        const double mh = d.mh_port[p];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[kMaxModes + m] += mh * (d.hprof[(long long)m * nh + p] * v);
    }
    // the port-plane data of this thread's first edge, read before the
    // barriers (none of it depends on this step's modal values)
    double ep0[kMaxModes], vp0[kMaxModes];
    long long pe0 = 0;
    double me0 = 0.0, cl0 = 0.0, cr0 = 0.0, csa0 = 0.0, csb0 = 0.0, ei0 = 0.0;
    const int p0 = split ? ne : threadIdx.x;
    double* cstate = d.comp_state + (long long)b * 2 * ne;
    if (p0 < ne) {
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m) {
            ep0[m] = m < M ? d.eprof[(long long)m * ne + p0] : 0.0;
            vp0[m] = m < M ? d.vprof[(long long)m * ne + p0] : 0.0;
        }
        pe0 = d.port_e[p0];
        me0 = d.me_port[p0];
        ei0 = eint[p0];
        if (d.comp_on) {
            cl0 = d.comp_live[p0];
            cr0 = d.comp_r[p0];
            csa0 = cstate[p0];
            csb0 = cstate[ne + p0];
        }
    }
    if (!split) block_sum_modes<false>(acc, M, red, wred);  // ends with a block barrier (s_conv too)
    const double i_sum = split && threadIdx.x < M ? red[M + threadIdx.x] : 0.0;
    __syncthreads();

    // 3. Per-mode boundary value: one thread per mode (the modes' scalar
    //    float64 recursions are independent of each other).
    if (threadIdx.x < M) {
        const int m = threadIdx.x;
        const double vin = red[m];
        s_vint[m] = vin;
        double vc = vint0 + mur * (vin - vport0);
        if (m == exc && !dtbc) {
            const double scat_int_now = vin - inc_int_now;
            const double scat_int_prev = vint0 - inc_int_prev;
            const double scat_face_prev = vport0 - inc_face_prev;
            vc = src_new + scat_int_prev + mur * (scat_int_now - scat_face_prev);
        }
        if (dtbc) {
            const double src = m == exc ? src_dtbc : 0.0;
            const double conv_w = s_conv[2 * m], u_inc = s_conv[2 * m + 1];
            const double ghost = src + conv_w;
            double* wh = d.whist + ((long long)b * M + m) * d.cap;
            double* sh = d.shist + ((long long)b * M + m) * d.cap;
            wh[n] = u0 - u_inc;
            sh[n] = src;
            double un = (2.0 - 2.0 * r2 - q2) * u0;
            un = un - up0;
            un = un + r2 * (ghost + vint0);
            u_prev[m] = u0;
            u[m] = un;
            vc = un;
        }
        s_vc[m] = vc;
        if (split) {
            // the reconstruction runs in k_modal_scatter; the scalars that
            // need no plane sum are final here
            double* vals = d.vals + (long long)b * 2 * kMaxModes;
            vals[m] = vc;
            vals[kMaxModes + m] = vin;
            const long long r = ((long long)b * pa.rec.cap + n) * pa.rec.nch + d.channel0 + m;
            pa.rec.I[r] = i_sum * d.rec_scale[m];
            Vport_prev[m] = vc;
            Vint_prev[m] = vin;
            atomic_max_nonneg(pa.absmax + b, fmax(0.0, fabs(vc) * d.rec_scale[m]));
        }
    }
    if (split) return;  // uniform over the block
    __syncthreads();

    // 4. Reconstruct the port plane from the modal expansion (+ complement),
    //    and 5. the recorder's V samples of the corrected port plane, from the
    //    value each thread has just stored (acc[0..M)).
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) acc[m] = 0.0;
    auto edge = [&](int p, const double (&ep)[kMaxModes], const double (&vp)[kMaxModes], long long pe, double me,
                    double cl, double cr, double csa, double csb, double ei) {
        double v = 0.0;
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) v += s_vc[m] * ep[m];
        if (d.comp_on) {
            double ci = ei;
#pragma unroll
            for (int m = 0; m < kMaxModes; ++m)
                if (m < M) ci -= s_vint[m] * ep[m];
            const double cp = cl * (csa + cr * (ci - csb));
            v += cp;
            cstate[p] = ci;
            cstate[ne + p] = cp;
        }
        enew[p] = v;
        const T stored = (T)v;
        E[pe] = stored;
        const double vr = (double)stored;
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[m] += me * (vp[m] * vr);
    };
    if (p0 < ne) edge(p0, ep0, vp0, pe0, me0, cl0, cr0, csa0, csb0, ei0);
    for (int p = p0 + blockDim.x; p < ne; p += blockDim.x) {
        double ep[kMaxModes], vp[kMaxModes];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m) {
            ep[m] = m < M ? d.eprof[(long long)m * ne + p] : 0.0;
            vp[m] = m < M ? d.vprof[(long long)m * ne + p] : 0.0;
        }
        const bool c = d.comp_on != 0;
        edge(p, ep, vp, d.port_e[p], d.me_port[p], c ? d.comp_live[p] : 0.0, c ? d.comp_r[p] : 0.0,
             c ? cstate[p] : 0.0, c ? cstate[ne + p] : 0.0, eint[p]);
    }
    block_sum_modes<true>(acc, M, red, wred);
    if (threadIdx.x < M) {
        const int m = threadIdx.x;
        const long long r = ((long long)b * pa.rec.cap + n) * pa.rec.nch + d.channel0 + m;
        pa.rec.V[r] = red[m] * d.rec_scale[m];
        pa.rec.I[r] = red[M + m] * d.rec_scale[m];
        Vport_prev[m] = s_vc[m];
        Vint_prev[m] = s_vint[m];
        // fmax drops a NaN as the serial max over the modes did
        atomic_max_nonneg(pa.absmax + b, fmax(0.0, fabs(s_vc[m]) * d.rec_scale[m]));
    }
}

// Large planes, before k_modal: chunk blockIdx.x of the port's edges and
// faces: the interior-plane samples into the scratch and the partial sums
// of the interior projection (modes 0..M) and of the recorder's I (M..2M).
template <typename T>
__global__ void __launch_bounds__(kPortThreads)
    k_modal_gather(const T* __restrict__ e, const T* __restrict__ h, PortsArgs pa, const ModalDev* __restrict__ ports) {
    const ModalDev& d = ports[blockIdx.y];
    const int c = blockIdx.x, b = blockIdx.z;
    if (d.n_chunks <= 1 || c >= d.n_chunks) return;  // uniform over the block
    const int M = d.n_modes, ne = d.n_e, nh = d.n_h;
    const T* E = e + (long long)b * pa.e_block;
    const T* H = h + (long long)b * pa.h_block;
    double* eint = d.scratch + (long long)b * 2 * ne;
    __shared__ double red[2 * kMaxModes];
    __shared__ double wred[kPortThreads / 32][2 * kMaxModes];
    double acc[2 * kMaxModes];
#pragma unroll
    for (int m = 0; m < 2 * kMaxModes; ++m) acc[m] = 0.0;
    const int e1 = min(ne, (c + 1) * d.chunk), h1 = min(nh, (c + 1) * d.chunk);
    for (int p = c * d.chunk + threadIdx.x; p < e1; p += blockDim.x) {
        const double v = (double)E[d.int_e[p]];
        eint[p] = v;
        const double me = d.me_int[p];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[m] += me * (d.vprof[(long long)m * ne + p] * v);
    }
    for (int p = c * d.chunk + threadIdx.x; p < h1; p += blockDim.x) {
        const double v = (double)H[d.port_h[p]];
        const double mh = d.mh_port[p];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[kMaxModes + m] += mh * (d.hprof[(long long)m * nh + p] * v);
    }
    block_sum_modes<true>(acc, M, red, wred);
    if (threadIdx.x < 2 * M)
        d.part[((long long)b * d.n_chunks + c) * 2 * kMaxModes + threadIdx.x] = red[threadIdx.x];
}

// Large planes, after k_modal: chunk blockIdx.x of the port plane rebuilt
// from the step's boundary values (+ complement), and the partial sums of
// the recorder's V; the last CTA of the (port, field set) to finish adds
// the partials in chunk order and writes the V samples.
template <typename T>
__global__ void __launch_bounds__(kPortThreads)
    k_modal_scatter(T* __restrict__ e, PortsArgs pa, const ModalDev* __restrict__ ports) {
    const ModalDev& d = ports[blockIdx.y];
    const int c = blockIdx.x, b = blockIdx.z;
    if (d.n_chunks <= 1 || c >= d.n_chunks) return;  // uniform over the block
    const int M = d.n_modes, ne = d.n_e;
    const long long n = *pa.step;
    T* E = e + (long long)b * pa.e_block;
    double* enew = d.scratch + (long long)b * 2 * ne + ne;
    const double* eint = d.scratch + (long long)b * 2 * ne;
    double* cstate = d.comp_state + (long long)b * 2 * ne;
    __shared__ double red[2 * kMaxModes];
    __shared__ double wred[kPortThreads / 32][2 * kMaxModes];
    __shared__ double s_vc[kMaxModes], s_vint[kMaxModes];
    __shared__ int s_last;
    if (threadIdx.x < M) {
        s_vc[threadIdx.x] = d.vals[(long long)b * 2 * kMaxModes + threadIdx.x];
        s_vint[threadIdx.x] = d.vals[(long long)b * 2 * kMaxModes + kMaxModes + threadIdx.x];
    }
    __syncthreads();
    double acc[2 * kMaxModes];
#pragma unroll
    for (int m = 0; m < 2 * kMaxModes; ++m) acc[m] = 0.0;
    const int e1 = min(ne, (c + 1) * d.chunk);
    for (int p = c * d.chunk + threadIdx.x; p < e1; p += blockDim.x) {
        double ep[kMaxModes];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m) ep[m] = m < M ? d.eprof[(long long)m * ne + p] : 0.0;
        double v = 0.0;
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) v += s_vc[m] * ep[m];
        if (d.comp_on) {
            double ci = eint[p];
#pragma unroll
            for (int m = 0; m < kMaxModes; ++m)
                if (m < M) ci -= s_vint[m] * ep[m];
            const double cp = d.comp_live[p] * (cstate[p] + d.comp_r[p] * (ci - cstate[ne + p]));
            v += cp;
            cstate[p] = ci;
            cstate[ne + p] = cp;
        }
        enew[p] = v;
        const T stored = (T)v;
        E[d.port_e[p]] = stored;
        const double vr = (double)stored, me = d.me_port[p];
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
            if (m < M) acc[m] += me * (d.vprof[(long long)m * ne + p] * vr);
    }
    block_sum_modes<false>(acc, M, red, wred);
    double* part = d.part + (long long)pa.B * d.n_chunks * 2 * kMaxModes;  // V partials after the gather area
    if (threadIdx.x < M) part[((long long)b * d.n_chunks + c) * kMaxModes + threadIdx.x] = red[threadIdx.x];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(d.done + b, 1) == d.n_chunks - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x < M) {
        const int m = threadIdx.x;
        double a = 0.0;
        for (int q = 0; q < d.n_chunks; ++q) a += __ldcg(part + ((long long)b * d.n_chunks + q) * kMaxModes + m);
        const long long r = ((long long)b * pa.rec.cap + n) * pa.rec.nch + d.channel0 + m;
        pa.rec.V[r] = a * d.rec_scale[m];
    }
    if (threadIdx.x == 0) d.done[b] = 0;
}

// Partial DTBC convolutions of the coming update at chain step n (the
// step counter): chunk c of the history, i in [c K, (c + 1) K) and i < n,
// of every DTBC mode of port blockIdx.z, field set blockIdx.y, with the
// kernel table in effect at step n (auto-extended by doubling,
// dtbc.py:351-363, dtbc.py:417-463).  Only history before step n is read,
// so this runs beside the stencil of the same step.
constexpr int kConvThreads = 128;

__global__ void __launch_bounds__(kConvThreads) k_dtbc_conv(PortsArgs pa, const ModalDev* __restrict__ ports) {
    const ModalDev& d = ports[blockIdx.z];
    const int b = blockIdx.y, c = blockIdx.x;
    const long long n = *pa.step;
    const long long lo = (long long)c * kConvChunk;
    if (c >= d.conv_chunks || lo >= n) return;
    const long long hi = min(lo + kConvChunk, n);
    const int M = d.n_modes;
    long long tlen = d.n0;
    long long toff = 0;
    while (tlen < n + 1) {
        toff += tlen;
        tlen *= 2;
    }
    __shared__ double wsum[kConvThreads / 32][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int m = 0; m < M; ++m) {
        if (!d.is_dtbc[m]) continue;
        const double* lt = d.ktab[m] + toff;
        const double* wh = d.whist + ((long long)b * M + m) * d.cap;
        const double* sh = d.shist + ((long long)b * M + m) * d.cap;
        double aw = 0.0, as = 0.0;
        for (long long i = lo + threadIdx.x; i < hi; i += kConvThreads) {
            const double l = lt[n - i];
            aw += l * wh[i];
            as += l * sh[i];
        }
        for (int o = 16; o > 0; o >>= 1) {
            aw += __shfl_xor_sync(0xffffffffu, aw, o);
            as += __shfl_xor_sync(0xffffffffu, as, o);
        }
        if (lane == 0) {
            wsum[warp][0] = aw;
            wsum[warp][1] = as;
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            double a = 0.0;
            for (int w = 0; w < kConvThreads / 32; ++w) a += wsum[w][threadIdx.x];
            d.conv[(((long long)b * M + m) * d.conv_chunks + c) * 2 + threadIdx.x] = a;
        }
        __syncthreads();
    }
}

}  // namespace

void launch_dtbc_conv(const PortsArgs& pa, const ModalDev* d, int n_modal, int max_chunks, cudaStream_t s) {
    if (n_modal <= 0 || max_chunks <= 0) return;
    k_dtbc_conv<<<dim3(max_chunks, pa.B, n_modal), kConvThreads, 0, s>>>(pa, d);
}

template <typename T>
void launch_lumped(T* e, const PortsArgs& pa, const LumpedDev* d, int n_lumped, cudaStream_t s) {
    if (n_lumped <= 0) return;
    k_lumped<T><<<dim3(n_lumped, pa.B), 32, 0, s>>>(e, pa, d);
}

template <typename T>
void launch_modal(T* e, const T* h, const PortsArgs& pa, const ModalDev* d, int n_modal, int max_chunks,
                  cudaStream_t s) {
    if (n_modal <= 0) return;
    if (max_chunks > 1) k_modal_gather<T><<<dim3(max_chunks, n_modal, pa.B), kPortThreads, 0, s>>>(e, h, pa, d);
    k_modal<T><<<dim3(n_modal, pa.B), kPortThreads, 0, s>>>(e, h, pa, d);
    if (max_chunks > 1) k_modal_scatter<T><<<dim3(max_chunks, n_modal, pa.B), kPortThreads, 0, s>>>(e, pa, d);
}

template void launch_lumped<float>(float*, const PortsArgs&, const LumpedDev*, int, cudaStream_t);
template void launch_lumped<double>(double*, const PortsArgs&, const LumpedDev*, int,
                                    cudaStream_t);
template void launch_modal<float>(float*, const float*, const PortsArgs&, const ModalDev*, int, int,
                                  cudaStream_t);
template void launch_modal<double>(double*, const double*, const PortsArgs&, const ModalDev*, int, int,
                                   cudaStream_t);

}  // namespace fitb
