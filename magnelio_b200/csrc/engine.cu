// Host side of the FIT-TD engine: handle lifetime, uploads, the per-step
// launch sequence captured into CUDA graphs, readback and checkpointing.
// Implements the C ABI declared in include/fitb200.h.
//
// One leapfrog step (reference loop body: src/magnelio/solver/fit_td.py
// :950-1007) is the launch sequence
//   update_E (+ CPML psi_E)         fit_td.py:843-876
//   modal ports, lumped ports       fit_td.py:975-976 (+ recorder :981-982)
//   update_H (+ CPML psi_H)         fit_td.py:893-920
//   DFT stage / flush per monitor   fit_td.py:1001-1002
//   step counter advance
// PEC faces are folded into the coefficients by the caller (alpha_E = beta_E
// = 0 on their tangential edges), which holds them at exact +0.0 the way the
// reference's frozen PEC edges are (fit_td.py:497-513).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fitb200.h"
#include "fitb_common.cuh"

namespace fitb {

namespace {

thread_local std::string g_last_error;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw Error(code, buf);
}

void ck(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(FITB_ERR_NOMEM, "%s: %s", what, cudaGetErrorString(e));
    }
    fail(FITB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Owning device buffer.
// Setup copies and fills below run on the legacy default stream, which the
// handles' non-blocking streams do not wait for, and a pageable host-to-
// device cudaMemcpy may return before its DMA lands: each one is finished
// (legacy_sync) before the function that issued it returns, so no kernel on
// a handle's stream can read a table that is still being written.
inline void legacy_sync(const char* what) { ck(cudaStreamSynchronize(0), what); }

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t n, bool zero = true) {
        release();
        if (n == 0) return;
        ck(cudaMalloc(&p, n), "cudaMalloc");
        bytes = n;
        if (zero) {
            ck(cudaMemset(p, 0, n), "cudaMemset");
            legacy_sync("cudaMemset sync");
        }
    }
    template <typename U>
    U* as() const {
        return static_cast<U*>(p);
    }
};

// Page-locked host memory, grown on demand: small device-to-host reads (the
// V/I of a step and the pipeline status word) land here as one batch of
// stream-ordered copies behind a single synchronisation.
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() {
        if (p) cudaFreeHost(p);
    }
    void reserve(size_t n) {
        if (n <= bytes) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        ck(cudaMallocHost(&p, n), "cudaMallocHost");
        bytes = n;
    }
};

template <typename U>
void upload(DevBuf& d, const std::vector<U>& v) {
    d.alloc(v.size() * sizeof(U), false);
    if (!v.empty()) {
        ck(cudaMemcpy(d.p, v.data(), v.size() * sizeof(U), cudaMemcpyHostToDevice), "upload");
        legacy_sync("upload sync");
    }
}

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

struct FaceHost {
    int face = 0;
    bool pec = false;  // some air mask entry is 0
    FaceDev dev{};
    DevBuf psi, air, bcc;
    DevBuf psi2;  // the fused step's second psi buffer
};

struct LumpedHost {
    LumpedDev dev{};
    std::vector<long long> off_host;  // E offsets the element writes
    DevBuf off, sign, beta, src, st;
    std::vector<double> src_host;  // [B][n_src]
};

// ADE dispersion of one side: host copies of every block, merged into the
// device tables on each addition.
struct DispHost {
    DispDev dev{};
    std::vector<long long> off, slot;
    std::vector<double> g;
    std::vector<int> state_block, pole_start{0}, kind;
    std::vector<double> k_re, k_im, c_re, c_im, opk_re, opk_im, hw;
    long long n_slots = 0;
    DevBuf d_off, d_g, d_state_block, d_slot, d_J, d_fprev, d_pole_start, d_kind, d_k_re, d_k_im, d_c_re, d_c_im,
        d_opk_re, d_opk_im, d_hw, d_uoff, d_ustart, d_ustate;
    bool present() const { return !off.empty(); }
};

struct SibcHost {
    SibcDev dev{};
    std::vector<long long> off, slot;
    std::vector<double> g, k, q, hopk;
    std::vector<int> state_block, br_start{0};
    long long n_slots = 0;
    DevBuf d_off, d_g, d_state_block, d_slot, d_u, d_hprev, d_br_start, d_k, d_q, d_hopk, d_uoff, d_ustart, d_ustate;
    bool present() const { return !off.empty(); }
};

struct PlaneWaveHost {
    PlaneWaveDev dev{};
    DevBuf e_off, e_start, e_coef, e_delay, h_off, h_start, h_coef, h_delay, scale;
    std::vector<double> scale_host;
    std::vector<long long> e_off_host;  // E offsets it writes (fused-step fix-up)
};

struct ModalHost {
    ModalDev dev{};
    std::vector<long long> port_e_host;  // E offsets the port writes
    int n_modes = 0;
    DevBuf port_e, int_e, port_h, me_port, me_int, mh_port, eprof, vprof, hprof;
    DevBuf comp_r, comp_live;
    DevBuf st, whist, shist, comp_state, scratch, exc, wf, buflen;
    DevBuf conv;  // DTBC convolution partials of the current step
    DevBuf part, vals, done;  // the chunked path of a large plane
    std::vector<std::vector<double>> ktabs;  // per mode: concatenated tables
    std::vector<int> n_tables_mode;
    std::vector<double> dtbc_r, dtbc_q;      // per mode: the DTBC chain parameters
    DevBuf ktab[kMaxModes];
    std::vector<int> exc_host, buflen_host;
    std::vector<double> wf_host;  // [B][n_wf]
    long long n_wf = 0;
};

struct BandHost {
    BandDev dev{};
    int p = 0;
    DevBuf eu, ev, x1, hh, Wu, Wv, Mc, D0, Dm1, me, vprof, mh, hprof, rec_scale;
    DevBuf kout, kin, st, x1prev, whist, shist, src, src_on, conv;
    std::vector<double> kout_host, kin_host;  // tables one after the other
    int n_out = 0, n_in = 0;                  // tables set
    std::vector<double> src_host;             // [B][n_src][p]
    std::vector<int> src_on_host;
    long long n_src = 0;
};

struct DftHost {
    DftDev dev{};
    DevBuf omega, inv, dual, stage, wst, bins, cmp, base;
    long long base_host = 0;
    std::vector<int> comps;
    int i0, i1, j0, j1, k0, k1;
};

constexpr int kModeSimple = 0, kModeStream = 1, kModeBulk = 2, kModeVec = 3, kModeFused = 4;

}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

struct Handle {
    fitb_desc desc{};
    int prec = 4;
    size_t esz = 4;
    Geom g{};
    int B = 1;
    double dt = 0.0;
    cudaStream_t stream = nullptr;
    // second stream of the step graphs: the DTBC convolutions run on it
    // beside the stencil (fork / join by events inside the capture)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // the slab step's CPML unit lists, one stream each beside the CPML-free
    // list on the handle's stream
    cudaStream_t slab_side[kSlabLists] = {};
    cudaEvent_t ev_sfork = nullptr, ev_sjoin[kSlabLists] = {};
    // completion tickets of asynchronous reads (fitb_read_vi_async): a ring
    static constexpr int kTickets = 64;
    cudaEvent_t tickets[kTickets] = {};
    long long next_ticket = 0;
    DevBuf e, h, aE, bE, aH, bH, meps, mmu, staging;
    // Fused step: second field buffers; `cur` names the buffer set that
    // holds the current fields (always 0 for the in-place kernels).
    DevBuf e2, h2;
    int cur = 0;
    DevBuf fix_cells;  // int4 (i, j, k, 0): H cells next to port-written E edges
    int n_fix = 0;
    // Slab form of the fused step: unit lists by CPML face-slot count
    DevBuf slab_units[kSlabLists];
    int n_slab_units[kSlabLists] = {};
    // Dead units left out of the slab step's lists (their cells need the
    // buffer-set sync before the next step after any host write of fields)
    DevBuf slab_dead;
    int n_slab_dead = 0;
    bool skip_sync = false;
    std::vector<int4> fix_host;  // H cells next to port-written E edges (host copy)
    bool coeffs_set = false;
    std::vector<std::unique_ptr<FaceHost>> faces;
    std::vector<std::unique_ptr<LumpedHost>> lumped;
    std::vector<std::unique_ptr<ModalHost>> modal;
    int modal_chunks = 1;  // the largest chunk count of the modal ports
    std::vector<std::unique_ptr<DftHost>> dft;
    std::vector<std::unique_ptr<PlaneWaveHost>> pws;
    DispHost disp[2];  // E side, H side
    SibcHost sibc;     // surface-impedance walls (H side)
    std::vector<std::unique_ptr<BandHost>> band;  // band-subspace DTBC ports
    DevBuf d_band;
    DevBuf d_lumped, d_modal, d_dft;
    int dft_stage_blocks = 0, dft_flush_blocks = 0;
    size_t dft_flush_smem = 0;
    DevBuf ticket;  // CTA completion counter of the merged flush launch
    int launches_per_step = 0;
    bool port_tables_dirty = true;
    DevBuf step;          // long long
    long long steps_done = 0;
    DevBuf recV, recI;    // [B][cap][nch]
    long long cap = 0;
    int nch = 0;
    DevBuf absmax;        // [B]
    DevBuf energy_partials, energy_out;
    int energy_blocks = 1184;
    cudaGraphExec_t graph_chunk[2] = {nullptr, nullptr};  // per starting buffer set
    cudaGraphExec_t graph_one[2] = {nullptr, nullptr};
    int chunk = 16;
    bool graphs_valid = false;
    long long launches = 0;
    int ichunk = 16;
    // Bulk-copy pipelined stencil (single field set); status word of its
    // bounded waits.
    BulkPlan plan{};
    int stencil_mode = 0;  // kModeSimple / kModeStream / kModeBulk / kModeVec
    int vec_variant = 0;   // vector width x register cap of the vec kernels
    int stream_variant = 0;  // register cap of the stream kernels
    int fused_variant = 0; // kernel form of the fused step (stencil_fused.cu)
    StreamPlan splan{};
    DevBuf status;
    HostBuf host_io;  // pinned landing area of fitb_read_vi
    // Compact coefficient storage of the stream kernels (kCoefF16 /
    // kCoefBF16): {aE, bE, aH, bH} as 16-bit [3][vol] with power-of-two
    // scales cs[4 * array + component]; coef_max holds the per-component
    // max |x| of the last upload.
    int coef_kind = 0;
    DevBuf cq[4];
    float cs[16] = {};
    double coef_max[4][3] = {};

    ~Handle() {
        for (int q = 0; q < 2; ++q) {
            if (graph_chunk[q]) cudaGraphExecDestroy(graph_chunk[q]);
            if (graph_one[q]) cudaGraphExecDestroy(graph_one[q]);
        }
        if (ev_sfork) cudaEventDestroy(ev_sfork);
        for (auto& t : tickets)
            if (t) cudaEventDestroy(t);
        for (int q = 0; q < kSlabLists; ++q) {
            if (ev_sjoin[q]) cudaEventDestroy(ev_sjoin[q]);
            if (slab_side[q]) cudaStreamDestroy(slab_side[q]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
    bool any_dtbc() const {
        for (auto& mp : modal)
            for (int m = 0; m < mp->n_modes; ++m)
                if (mp->dev.is_dtbc[m]) return true;
        return false;
    }

    long long e_block() const { return 3 * g.vol; }
    DevBuf& Ec() { return cur ? e2 : e; }
    DevBuf& Hc() { return cur ? h2 : h; }
    DevBuf& En() { return cur ? e : e2; }
    DevBuf& Hn() { return cur ? h : h2; }
    long long nE() const {
        return (long long)g.nx * (g.ny + 1) * (g.nz + 1) + (long long)(g.nx + 1) * g.ny * (g.nz + 1) +
               (long long)(g.nx + 1) * (g.ny + 1) * g.nz;
    }
    long long nH() const {
        return (long long)(g.nx + 1) * g.ny * g.nz + (long long)g.nx * (g.ny + 1) * g.nz +
               (long long)g.nx * g.ny * (g.nz + 1);
    }
    long long comp_size(int c) const {
        int ni, nj, nk;
        comp_shape(g, c, ni, nj, nk);
        return (long long)ni * nj * nk;
    }
    // Flat reference index (within E or H vector) -> offset into the padded
    // field-set block (component * vol + padded index).
    long long flat_to_off(bool is_h, long long flat) const {
        int c0 = is_h ? 3 : 0;
        long long rem = flat;
        for (int q = 0; q < 3; ++q) {
            long long sz = comp_size(c0 + q);
            if (rem < sz) {
                int ni, nj, nk;
                comp_shape(g, c0 + q, ni, nj, nk);
                int k = (int)(rem % nk);
                long long r = rem / nk;
                int j = (int)(r % nj);
                int i = (int)(r / nj);
                return (long long)q * g.vol + pidx(g, i, j, k);
            }
            rem -= sz;
        }
        fail(FITB_ERR_ARG, "flat index %lld out of range for %s (size %lld)", flat, is_h ? "H" : "E",
             is_h ? nH() : nE());
    }
};

}  // namespace fitb

struct fitb_handle {
    fitb::Handle impl;
};

using fitb::fail;
using fitb::ck;

namespace fitb {
namespace {

void check_device_status(Handle& H);

template <typename T>
std::vector<T> cast_vec(const double* src, long long n) {
    std::vector<T> v((size_t)n);
    for (long long q = 0; q < n; ++q) v[(size_t)q] = (T)src[q];
    return v;
}

// Upload a host array in the reference flat layout (three components,
// starting at component c0) into a padded [3][vol] device array.
template <typename T>
void pack3(Handle& H, const T* host_flat, T* dev_padded, int c0) {
    long long n = (c0 == 0) ? H.nE() : H.nH();
    ck(cudaMemcpyAsync(H.staging.p, host_flat, (size_t)n * sizeof(T), cudaMemcpyHostToDevice, H.stream),
       "H2D staging");
    long long off = 0;
    for (int q = 0; q < 3; ++q) {
        launch_pack<T>(H.staging.as<T>(), dev_padded + (long long)q * H.g.vol, H.g, c0 + q, off, H.stream);
        H.launches++;
        off += H.comp_size(c0 + q);
    }
    ck(cudaGetLastError(), "pack");
    ck(cudaStreamSynchronize(H.stream), "pack sync");
}

template <typename T>
void unpack3(Handle& H, const T* dev_padded, T* host_flat, int c0) {
    long long n = (c0 == 0) ? H.nE() : H.nH();
    long long off = 0;
    for (int q = 0; q < 3; ++q) {
        launch_unpack<T>(dev_padded + (long long)q * H.g.vol, H.staging.as<T>(), H.g, c0 + q, off, H.stream);
        H.launches++;
        off += H.comp_size(c0 + q);
    }
    ck(cudaGetLastError(), "unpack");
    ck(cudaMemcpyAsync(host_flat, H.staging.p, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost, H.stream),
       "D2H staging");
    ck(cudaStreamSynchronize(H.stream), "unpack sync");
    check_device_status(H);
}

// Device bytes the handle holds (every buffer it allocated).
size_t device_bytes(const Handle& H) {
    size_t n = 0;
    for (const DevBuf* d : {&H.e, &H.h, &H.e2, &H.h2, &H.aE, &H.bE, &H.aH, &H.bH, &H.meps, &H.mmu, &H.staging,
                            &H.fix_cells, &H.d_lumped, &H.d_modal, &H.d_dft, &H.ticket, &H.step, &H.recV, &H.recI,
                            &H.absmax, &H.energy_partials, &H.energy_out, &H.status})
        n += d->bytes;
    for (const auto& q : H.cq) n += q.bytes;
    for (const auto& f : H.faces) n += f->psi.bytes + f->psi2.bytes + f->air.bytes + f->bcc.bytes;
    for (const auto& l : H.lumped) n += l->off.bytes + l->sign.bytes + l->beta.bytes + l->src.bytes + l->st.bytes;
    for (const auto& m : H.modal) {
        for (const DevBuf* d : {&m->port_e, &m->int_e, &m->port_h, &m->me_port, &m->me_int, &m->mh_port, &m->eprof,
                                &m->vprof, &m->hprof, &m->comp_r, &m->comp_live, &m->st, &m->whist, &m->shist,
                                &m->comp_state, &m->scratch, &m->exc, &m->wf, &m->buflen, &m->part, &m->vals,
                                &m->done})
            n += d->bytes;
        for (const auto& k : m->ktab) n += k.bytes;
    }
    for (const auto& m : H.dft)
        for (const DevBuf* d : {&m->omega, &m->inv, &m->dual, &m->stage, &m->wst, &m->bins, &m->cmp, &m->base})
            n += d->bytes;
    for (const auto& w : H.pws)
        for (const DevBuf* d : {&w->e_off, &w->e_start, &w->e_coef, &w->e_delay, &w->h_off, &w->h_start, &w->h_coef,
                                &w->h_delay, &w->scale})
            n += d->bytes;
    for (const auto& D : H.disp)
        for (const DevBuf* d : {&D.d_off, &D.d_g, &D.d_state_block, &D.d_slot, &D.d_J, &D.d_fprev, &D.d_pole_start,
                                &D.d_kind, &D.d_k_re, &D.d_k_im, &D.d_c_re, &D.d_c_im, &D.d_opk_re, &D.d_opk_im,
                                &D.d_hw, &D.d_uoff, &D.d_ustart, &D.d_ustate})
            n += d->bytes;
    {
        const SibcHost& S = H.sibc;
        for (const DevBuf* d : {&S.d_off, &S.d_g, &S.d_state_block, &S.d_slot, &S.d_u, &S.d_hprev, &S.d_br_start,
                                &S.d_k, &S.d_q, &S.d_hopk, &S.d_uoff, &S.d_ustart, &S.d_ustate})
            n += d->bytes;
    }
    return n;
}

void invalidate_graphs(Handle& H) {
    for (int q = 0; q < 2; ++q) {
        if (H.graph_chunk[q]) cudaGraphExecDestroy(H.graph_chunk[q]);
        if (H.graph_one[q]) cudaGraphExecDestroy(H.graph_one[q]);
        H.graph_chunk[q] = H.graph_one[q] = nullptr;
    }
    H.graphs_valid = false;
}

// Recorder and DTBC history capacity (steps).  Growth keeps the contents
// and invalidates the captured graphs (they hold the old pointers).
void ensure_capacity(Handle& H, long long need) {
    if (need <= H.cap) return;
    // steps still running on the handle's stream write the old histories
    ck(cudaStreamSynchronize(H.stream), "capacity sync");
    long long ncap = std::max(need, std::max<long long>(2 * H.cap, 1024));
    if (H.nch > 0) {
        for (DevBuf* buf : {&H.recV, &H.recI}) {
            DevBuf nb;
            nb.alloc((size_t)H.B * ncap * H.nch * sizeof(double));
            if (buf->p && H.cap > 0)
                ck(cudaMemcpy2D(nb.p, (size_t)ncap * H.nch * sizeof(double), buf->p,
                                (size_t)H.cap * H.nch * sizeof(double), (size_t)H.cap * H.nch * sizeof(double),
                                H.B, cudaMemcpyDeviceToDevice),
                   "grow recorder");
            std::swap(buf->p, nb.p);
            std::swap(buf->bytes, nb.bytes);
        }
    }
    for (auto& mp : H.modal) {
        int M = mp->n_modes;
        mp->conv.alloc((size_t)H.B * M * ((ncap + kConvChunk - 1) / kConvChunk) * 2 * sizeof(double));
        for (DevBuf* buf : {&mp->whist, &mp->shist}) {
            DevBuf nb;
            nb.alloc((size_t)H.B * M * ncap * sizeof(double));
            if (buf->p && H.cap > 0)
                ck(cudaMemcpy2D(nb.p, (size_t)ncap * sizeof(double), buf->p, (size_t)H.cap * sizeof(double),
                                (size_t)H.cap * sizeof(double), (size_t)H.B * M, cudaMemcpyDeviceToDevice),
                   "grow DTBC history");
            std::swap(buf->p, nb.p);
            std::swap(buf->bytes, nb.bytes);
        }
    }
    for (auto& bp : H.band) {
        const int p = bp->p;
        bp->conv.alloc((size_t)H.B * ((ncap + kConvChunk - 1) / kConvChunk) * 2 * p * sizeof(double));
        for (DevBuf* buf : {&bp->whist, &bp->shist}) {
            DevBuf nb;
            nb.alloc((size_t)H.B * ncap * p * sizeof(double));
            if (buf->p && H.cap > 0)
                ck(cudaMemcpy2D(nb.p, (size_t)ncap * p * sizeof(double), buf->p, (size_t)H.cap * p * sizeof(double),
                                (size_t)H.cap * p * sizeof(double), (size_t)H.B, cudaMemcpyDeviceToDevice),
                   "grow band history");
            std::swap(buf->p, nb.p);
            std::swap(buf->bytes, nb.bytes);
        }
    }
    legacy_sync("capacity copy sync");
    H.cap = ncap;
    H.port_tables_dirty = true;
    invalidate_graphs(H);
}

// H cells whose update reads an E edge that a port writes between the E and
// the H update: the H update of cell (i, j, k) reads E at (i, j, k),
// (i+1, j, k), (i, j+1, k) and (i, j, k+1).
void build_fix_cells(Handle& H) {
    std::vector<long long> keys;
    auto add_edge = [&](long long off) {
        const long long r = off % H.g.vol;  // drop the component
        const int i = (int)(r / H.g.si) - 2;
        const long long rr = r % H.g.si;
        const int j = (int)(rr / H.g.sj), k = (int)(rr % H.g.sj);
        const int cand[4][3] = {{i, j, k}, {i - 1, j, k}, {i, j - 1, k}, {i, j, k - 1}};
        for (auto& c : cand) {
            if (c[0] < 0 || c[0] > H.g.nx || c[1] < 0 || c[1] > H.g.ny || c[2] < 0 || c[2] > H.g.nz) continue;
            keys.push_back(pidx(H.g, c[0], c[1], c[2]));
        }
    };
    for (auto& lp : H.lumped)
        for (long long o : lp->off_host) add_edge(o);
    for (auto& mp : H.modal)
        for (long long o : mp->port_e_host) add_edge(o);
    for (auto& pw : H.pws)
        for (long long o : pw->e_off_host) add_edge(o);
    // the slab step with E-side dispersion: the ADE update corrects E after
    // the step kernel's H update, so the H cells next to dispersive edges
    // are recomputed like those next to port edges
    if (is_slab_variant(H.fused_variant))
        for (long long o : H.disp[0].off) add_edge(o);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    std::vector<int4> cells;
    cells.reserve(keys.size());
    for (long long key : keys) {
        const int i = (int)(key / H.g.si) - 2;
        const long long rr = key % H.g.si;
        cells.push_back(make_int4(i, (int)(rr / H.g.sj), (int)(rr % H.g.sj), 0));
    }
    H.fix_host = cells;
    if (cells.empty()) cells.push_back(make_int4(0, 0, 0, 0));  // keep a valid pointer
    upload(H.fix_cells, cells);
    H.n_fix = (int)keys.size();
}

void build_slab_units(Handle& H);

void refresh_port_tables(Handle& H) {
    if (!H.port_tables_dirty) return;
    // the tables below are re-allocated: no launch may still read the old ones
    ck(cudaStreamSynchronize(H.stream), "port tables sync");
    std::vector<LumpedDev> ld;
    for (auto& lp : H.lumped) ld.push_back(lp->dev);
    upload(H.d_lumped, ld);
    std::vector<ModalDev> md;
    for (auto& mp : H.modal) {
        ModalDev d = mp->dev;
        d.whist = mp->whist.as<double>();
        d.shist = mp->shist.as<double>();
        d.cap = H.cap;
        d.conv = mp->conv.as<double>();
        d.conv_chunks = (int)((H.cap + kConvChunk - 1) / kConvChunk);
        md.push_back(d);
    }
    upload(H.d_modal, md);
    std::vector<BandDev> bd;
    for (auto& bp : H.band) {
        BandDev d = bp->dev;
        d.whist = bp->whist.as<double>();
        d.shist = bp->shist.as<double>();
        d.cap = H.cap;
        d.conv = bp->conv.as<double>();
        d.conv_chunks = (int)((H.cap + kConvChunk - 1) / kConvChunk);
        d.kout = bp->kout.as<double>();
        d.kin = bp->kin.as<double>();
        d.has_in = bp->n_in > 0 ? 1 : 0;
        d.src = bp->src.as<double>();
        d.n_src = bp->n_src;
        d.src_on = bp->src_on.as<int>();
        bd.push_back(d);
    }
    upload(H.d_band, bd);
    // monitors: block ranges of the merged stage / flush launches
    std::vector<DftDev> dd;
    int sb = 0, fb = 0;
    size_t smem = 0;
    for (auto& m : H.dft) {
        DftDev d = m->dev;
        d.sblk0 = sb;
        d.sblk = dft_blocks((long long)d.ncomp * d.ncell);
        d.fblk0 = fb;
        d.fblk = dft_blocks((long long)H.B * d.ncomp * d.ncell);
        sb += d.sblk;
        fb += d.fblk;
        smem = std::max(smem, (size_t)d.K * 2 * d.nf * sizeof(float2));
        m->dev.sblk0 = d.sblk0;
        m->dev.sblk = d.sblk;
        m->dev.fblk0 = d.fblk0;
        m->dev.fblk = d.fblk;
        dd.push_back(d);
    }
    upload(H.d_dft, dd);
    if (H.stencil_mode == kModeFused) build_fix_cells(H);
    if (H.stencil_mode == kModeFused && is_slab_variant(H.fused_variant)) build_slab_units(H);
    H.dft_stage_blocks = sb;
    H.dft_flush_blocks = fb;
    H.dft_flush_smem = smem;
    H.port_tables_dirty = false;
}

template <typename T>
StencilArgs<T> stencil_args(Handle& H) {
    StencilArgs<T> a{};
    a.g = H.g;
    a.B = H.B;
    a.e = H.Ec().as<T>();
    a.h = H.Hc().as<T>();
    a.e_next = H.En().as<T>();
    a.h_next = H.Hn().as<T>();
    a.aE = H.aE.as<T>();
    a.bE = H.bE.as<T>();
    a.aH = H.aH.as<T>();
    a.bH = H.bH.as<T>();
    a.nfaces = (int)H.faces.size();
    for (int q = 0; q < a.nfaces; ++q) {
        a.f[q] = H.faces[q]->dev;
        if (H.cur) std::swap(a.f[q].psi, a.f[q].psi_next);
    }
    a.ichunk = H.ichunk;
    const bool slab = H.stencil_mode == kModeFused && is_slab_variant(H.fused_variant);
    a.coef_kind = (H.stencil_mode == kModeStream || H.stencil_mode == kModeVec || slab) ? H.coef_kind : kCoefNative;
    for (int q = 0; q < 4; ++q) a.cq[q] = H.cq[q].as<unsigned short>();
    for (int q = 0; q < 16; ++q) a.cs[q] = H.cs[q];
    return a;
}

// Per-component max |x| of one host array in the reference flat layout.
template <typename S>
void comp_max(const Handle& H, const S* flat, int c0, double out[3]) {
    long long off = 0;
    for (int q = 0; q < 3; ++q) {
        const long long n = H.comp_size(c0 + q);
        double m = 0.0;
        for (long long r = 0; r < n; ++r) m = std::max(m, std::fabs((double)flat[off + r]));
        out[q] = m;
        off += n;
    }
}

// Re-encode the four update-coefficient arrays in the compact 16-bit form.
// Each component gets the power-of-two scale that puts its largest
// magnitude in [2^13, 2^14): far from the float16 overflow (65504) and
// keeping values down to 2^-24 of the maximum out of the subnormal range.
void compact_coeffs(Handle& H) {
    if (H.coef_kind == kCoefNative || !H.coeffs_set) return;
    DevBuf* src[4] = {&H.aE, &H.bE, &H.aH, &H.bH};
    for (int a = 0; a < 4; ++a) {
        if (!H.cq[a].p) H.cq[a].alloc((size_t)3 * H.g.vol * sizeof(unsigned short));
        for (int c = 0; c < 3; ++c) {
            const double m = H.coef_max[a][c];
            const int e = (m > 0.0 && std::isfinite(m)) ? std::max(std::min(std::ilogb(m), 100), -100) : 13;
            const float inv = std::ldexp(1.0f, 13 - e);
            H.cs[4 * a + c] = std::ldexp(1.0f, e - 13);
            unsigned short* dst = H.cq[a].as<unsigned short>() + (long long)c * H.g.vol;
            if (H.prec == 4)
                launch_compact<float>(src[a]->as<float>() + (long long)c * H.g.vol, dst, H.g.vol, inv, H.coef_kind,
                                      H.stream);
            else
                launch_compact<double>(src[a]->as<double>() + (long long)c * H.g.vol, dst, H.g.vol, inv,
                                       H.coef_kind, H.stream);
            H.launches++;
        }
    }
    ck(cudaGetLastError(), "compact coefficients");
    ck(cudaStreamSynchronize(H.stream), "compact coefficients sync");
}

PortsArgs ports_args(Handle& H) {
    PortsArgs pa{};
    pa.B = H.B;
    pa.e_block = H.e_block();
    pa.h_block = H.e_block();
    pa.step = H.step.as<long long>();
    pa.dt_lumped = H.dt;
    pa.rec.V = H.recV.as<double>();
    pa.rec.I = H.recI.as<double>();
    pa.rec.nch = H.nch;
    pa.rec.cap = H.cap;
    pa.absmax = H.absmax.as<double>();
    return pa;
}

// Fused-step variants: 0-6 the register / cp.async forms (1 in float32
// only), kFusedTileBase + v the TMA tile forms whose shared memory fits.
bool fused_variant_ok(int prec, int v) {
    if (v >= 0 && v <= 6) return !(v == 1 && prec == 8);
    if (is_slab_variant(v))
        return prec == 4 ? slab_supported<float>(v - kFusedSlabBase) : slab_supported<double>(v - kFusedSlabBase);
    const int t = v - kFusedTileBase;
    if (t < 0 || t >= kTileVariants) return false;
    return prec == 4 ? tile_supported<float>(t) : tile_supported<double>(t);
}

cudaError_t prepare_fused_any(int prec, int v) {
    if (is_slab_variant(v))
        return prec == 4 ? prepare_slab<float>(v - kFusedSlabBase) : prepare_slab<double>(v - kFusedSlabBase);
    if (v >= kFusedTileBase)
        return prec == 4 ? prepare_tile<float>(v - kFusedTileBase) : prepare_tile<double>(v - kFusedTileBase);
    return prec == 4 ? prepare_fused<float>(v) : prepare_fused<double>(v);
}

// Unit lists of the slab form for the handle's faces and march depth.
bool slab_units_of(const Handle& H, int variant, int ichunk, std::vector<int4> out[kSlabLists]) {
    FaceDev f[kMaxFaces];
    const int nf = (int)H.faces.size();
    if (nf > kMaxFaces) return false;
    for (int q = 0; q < nf; ++q) f[q] = H.faces[q]->dev;
    const int v = variant - kFusedSlabBase;
    if (H.B % slab_nb_of(v) != 0) return false;
    if (!plan_slab_units(H.g, f, nf, slab_tj_of(v), ichunk, out)) return false;
    // units reaching both faces of an axis need the six-slot instance
    bool air = false;
    for (auto& fh : H.faces) air = air || fh->pec;
    return out[4].empty() || (H.prec == 4 ? slab_six_ok<float>(v, air) : slab_six_ok<double>(v, air));
}

// Dead-unit skipping of the slab step (reference: solver/_tile_skip.py,
// on by default, MAGNELIO_TILE_SKIP=0 turns it off there; FITB_TILE_SKIP=0
// here).  Like the reference it stays off with TF/SF plane waves (their H
// injection can drive faces the analysis calls curl-dead).  Only units
// without CPML are candidates (psi stays exact), and units holding a port-
// or source-written edge or its H neighbours stay live.
bool tile_skip_on(const Handle& H) {
    const char* e = getenv("FITB_TILE_SKIP");
    return !(e && std::string(e) == "0") && H.pws.empty() && !H.disp[0].present() && !H.disp[1].present();
}

// Whether no dispersive state lies in a CPML slab.  The slab step applies
// the CPML inside its kernel, before the ADE update of the same side; the
// reference applies the ADE update first (fit_td.py:833-874), so the two
// orders agree exactly when no entry takes both.
bool disp_clear_of_cpml(const Handle& H) {
    for (const DispHost& D : H.disp)
        for (long long off : D.off) {
            const long long r = off % H.g.vol;
            const int i = (int)(r / H.g.si) - 2;
            const long long rr = r % H.g.si;
            const int j = (int)(rr / H.g.sj), k = (int)(rr % H.g.sj);
            for (auto& f : H.faces) {
                const int c = f->dev.axis == 0 ? i : (f->dev.axis == 1 ? j : k);
                if (c >= f->dev.lo && c < f->dev.lo + f->dev.n) return false;
            }
        }
    return true;
}

void build_slab_units(Handle& H) {
    if ((H.disp[0].present() || H.disp[1].present()) && !disp_clear_of_cpml(H))
        fail(FITB_ERR_STATE, "the slab step takes dispersive materials only outside the CPML slabs");
    std::vector<int4> lists[kSlabLists];
    const int ichunk = H.splan.ichunk, tj = slab_tj_of(H.fused_variant - kFusedSlabBase);
    if (!slab_units_of(H, H.fused_variant, ichunk, lists))
        fail(FITB_ERR_STATE, "the slab step does not take this grid / CPML layout");
    std::vector<int4> dead;
    if (tile_skip_on(H) && !lists[0].empty()) {
        const int n = (int)lists[0].size();
        DevBuf du, fl;
        upload(du, lists[0]);
        fl.alloc((size_t)n * sizeof(int));
        if (H.prec == 4)
            slab_unit_liveness<float>(H.g, H.aE.as<float>(), H.bE.as<float>(), H.aH.as<float>(), H.bH.as<float>(), tj,
                                      ichunk, du.as<int4>(), n, fl.as<int>(), H.stream);
        else
            slab_unit_liveness<double>(H.g, H.aE.as<double>(), H.bE.as<double>(), H.aH.as<double>(),
                                       H.bH.as<double>(), tj, ichunk, du.as<int4>(), n, fl.as<int>(), H.stream);
        ck(cudaGetLastError(), "unit liveness launch");
        std::vector<int> flags((size_t)n);
        ck(cudaMemcpyAsync(flags.data(), fl.p, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, H.stream),
           "unit liveness D2H");
        ck(cudaStreamSynchronize(H.stream), "unit liveness sync");
        // units holding a port / source edge's H neighbours (the fix-up cells)
        for (const int4& c : H.fix_host)
            for (int q = 0; q < n; ++q) {
                const int4& u = lists[0][(size_t)q];
                const int k0 = (u.x & 0xffff) * 32, j0 = (u.x >> 16) * tj, i0 = u.y, i1 = u.z;
                if (c.x >= i0 - 1 && c.x <= i1 && c.y >= j0 - 1 && c.y <= j0 + tj && c.z >= k0 - 1 &&
                    c.z <= k0 + 32)
                    flags[(size_t)q] = 1;
            }
        std::vector<int4> live;
        for (int q = 0; q < n; ++q) (flags[(size_t)q] ? live : dead).push_back(lists[0][(size_t)q]);
        lists[0].swap(live);
    }
    for (int q = 0; q < kSlabLists; ++q) {
        H.n_slab_units[q] = (int)lists[q].size();
        if (lists[q].empty()) lists[q].push_back(make_int4(0, 0, 0, 0));  // keep a valid pointer
        upload(H.slab_units[q], lists[q]);
    }
    H.n_slab_dead = (int)dead.size();
    if (dead.empty()) dead.push_back(make_int4(0, 0, 0, 0));
    upload(H.slab_dead, dead);
    H.skip_sync = H.n_slab_dead > 0;
}

// Makes both buffer sets agree on the skipped units' cells (after a host
// write of fields or a new unit plan).
void sync_dead_units(Handle& H) {
    if (!H.skip_sync) return;
    H.skip_sync = false;
    if (H.stencil_mode != kModeFused || !is_slab_variant(H.fused_variant) || H.n_slab_dead == 0) return;
    const int tj = slab_tj_of(H.fused_variant - kFusedSlabBase);
    if (H.prec == 4)
        slab_dead_sync<float>(H.g, H.aH.as<float>(), H.bH.as<float>(), tj, H.splan.ichunk, H.slab_dead.as<int4>(),
                              H.n_slab_dead, H.B, H.Ec().as<float>(), H.Hc().as<float>(), H.En().as<float>(),
                              H.Hn().as<float>(), H.stream);
    else
        slab_dead_sync<double>(H.g, H.aH.as<double>(), H.bH.as<double>(), tj, H.splan.ichunk, H.slab_dead.as<int4>(),
                               H.n_slab_dead, H.B, H.Ec().as<double>(), H.Hc().as<double>(), H.En().as<double>(),
                               H.Hn().as<double>(), H.stream);
    ck(cudaGetLastError(), "dead unit sync launch");
}

// Grid of the stream / vec kernels for the handle's batch and coefficient
// storage (occupancy depends on the kernel instance).
void plan_stencil(Handle& H) {
    if (H.stencil_mode != kModeStream && H.stencil_mode != kModeVec && H.stencil_mode != kModeFused) return;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, H.desc.device);
    if (H.stencil_mode == kModeFused && is_slab_variant(H.fused_variant)) {
        const int v = H.fused_variant - kFusedSlabBase;
        const int occ = H.prec == 4 ? slab_occupancy<float>(v) : slab_occupancy<double>(v);
        H.splan = H.prec == 4 ? plan_slab<float>(H.g, sms, occ, H.B, v) : plan_slab<double>(H.g, sms, occ, H.B, v);
    } else if (H.stencil_mode == kModeFused && H.fused_variant >= kFusedTileBase) {
        const int v = H.fused_variant - kFusedTileBase;
        const int occ = H.prec == 4 ? tile_occupancy<float>(v) : tile_occupancy<double>(v);
        H.splan = H.prec == 4 ? plan_tile<float>(H.g, sms, occ, H.B, v) : plan_tile<double>(H.g, sms, occ, H.B, v);
    } else if (H.stencil_mode == kModeFused) {
        const int v = H.fused_variant;
        const int occ = H.prec == 4 ? fused_occupancy<float>(v) : fused_occupancy<double>(v);
        H.splan = plan_fused(H.g, sms, occ, H.B, fused_tj_of(v));
    } else if (H.stencil_mode == kModeStream) {
        const int occ = H.prec == 4 ? stream_occupancy<float>(H.B, H.coef_kind, H.stream_variant)
                                    : stream_occupancy<double>(H.B, H.coef_kind, H.stream_variant);
        H.splan = plan_stream(H.g, sms, occ, H.B);
    } else {
        const int occ = H.prec == 4 ? vec_occupancy<float>(H.vec_variant, H.coef_kind)
                                    : vec_occupancy<double>(H.vec_variant, H.coef_kind);
        H.splan = plan_vec(H.g, sms, occ, H.B, vec_width_of(H.prec, H.coef_kind ? 0 : H.vec_variant));
    }
}

// One launch of the E (which == 0) or H (which == 1) update, with the
// handle's kernel choice: the software-pipelined stencil for one field set,
// the bulk-copy pipeline on request, the batched kernel for B > 1.  A side
// with dispersive materials takes its CPML corrections in separate passes
// after the ADE update, so its stencil launch carries no faces.
template <typename T>
void launch_half(Handle& H, int which) {
    StencilArgs<T> sa = stencil_args<T>(H);
    if (H.disp[which].present() || (which == 1 && H.sibc.present())) sa.nfaces = 0;
    switch (H.stencil_mode) {
        case kModeStream:
            launch_stream_half<T>(sa, H.splan, H.stream_variant, which, H.stream);
            break;
        case kModeVec:
            launch_vec_half<T>(sa, H.splan, H.vec_variant, which, H.stream);
            break;
        case kModeBulk:
            which == 0 ? launch_update_E_bulk<T>(sa, H.plan, H.status.as<int>(), H.stream)
                       : launch_update_H_bulk<T>(sa, H.plan, H.status.as<int>(), H.stream);
            break;
        default:
            which == 0 ? launch_update_E<T>(sa, H.stream) : launch_update_H<T>(sa, H.stream);
    }
}

// The fused-step launch of the handle's variant (register / cp.async forms
// or the TMA tile form).
// (the tile form: the tile kernel and its E-side CPML passes).  Returns the
// launches issued.
template <typename T>
int launch_fused(Handle& H, const StencilArgs<T>& sa) {
    if (is_slab_variant(H.fused_variant)) {
        const int4* units[kSlabLists];
        bool air = false;
        for (int q = 0; q < kSlabLists; ++q) units[q] = H.slab_units[q].as<int4>();
        for (auto& f : H.faces) air = air || f->pec;
        // every CPML list runs on a stream of its own beside the CPML-free
        // list (disjoint units), all joined before anything reads the new
        // fields
        cudaStream_t streams[kSlabLists];
        streams[0] = H.stream;
        bool forked = false;
        for (int q = 1; q < kSlabLists; ++q) {
            streams[q] = H.n_slab_units[q] > 0 ? H.slab_side[q] : H.stream;
            if (H.n_slab_units[q] > 0 && !forked) {
                ck(cudaEventRecord(H.ev_sfork, H.stream), "slab fork record");
                forked = true;
            }
            if (H.n_slab_units[q] > 0) ck(cudaStreamWaitEvent(H.slab_side[q], H.ev_sfork, 0), "slab fork wait");
        }
        const int n = launch_slab_step<T>(sa, H.splan.ichunk, H.fused_variant - kFusedSlabBase, units,
                                          H.n_slab_units, air, H.status.as<int>(), streams);
        if (n == -4) fail(FITB_ERR_STATE, "the slab step variant has no kernel for this batch / unit list");
        if (n < 0) fail(FITB_ERR_CUDA, "tensor maps of the slab step could not be encoded");
        for (int q = 1; q < kSlabLists; ++q) {
            if (H.n_slab_units[q] <= 0) continue;
            ck(cudaEventRecord(H.ev_sjoin[q], H.slab_side[q]), "slab join record");
            ck(cudaStreamWaitEvent(H.stream, H.ev_sjoin[q], 0), "slab join wait");
        }
        return n;
    }
    if (H.fused_variant >= kFusedTileBase) {
        if (launch_tile_step<T>(sa, H.splan, H.fused_variant - kFusedTileBase, H.status.as<int>(), H.stream) != 0)
            fail(FITB_ERR_CUDA, "tensor maps of the tile step could not be encoded");
        const int ne = launch_tile_cpml_E<T>(sa, H.stream);
        if (ne < 0) fail(FITB_ERR_STATE, "the tile step does not take this grid / CPML layout");
        return 1 + ne;
    }
    launch_fused_step<T>(sa, H.splan, H.fused_variant, H.stream);
    return 1;
}

// The whole stencil part of a fused step (measurement helper: no ports).
int launch_fused_any(Handle& H) {
    if (H.prec == 4) {
        const StencilArgs<float> sa = stencil_args<float>(H);
        int n = launch_fused<float>(H, sa);
        if (is_tile_variant(H.fused_variant)) n += launch_tile_cpml_H<float>(sa, H.stream);
        return n;
    }
    const StencilArgs<double> sa = stencil_args<double>(H);
    int n = launch_fused<double>(H, sa);
    if (is_tile_variant(H.fused_variant)) n += launch_tile_cpml_H<double>(sa, H.stream);
    return n;
}

void launch_stencil_half(Handle& H, int which) {
    if (H.prec == 4)
        launch_half<float>(H, which);
    else
        launch_half<double>(H, which);
}

// After side `sd`'s stencil launch: the ADE history subtraction and pole
// advance, then that side's CPML faces in order (the reference's order,
// fit_td.py:833-874).  Returns the launches issued.
template <typename T>
int disp_complete(Handle& H, int sd) {
    const bool sibc = sd == 1 && H.sibc.present();
    if (!H.disp[sd].present() && !sibc) return 0;
    T* F = (sd == 0 ? H.Ec() : H.Hc()).as<T>();
    const T* beta = (sd == 0 ? H.bE : H.bH).as<T>();
    int n = 0;
    if (H.disp[sd].present()) {
        launch_disp_update<T>(F, H.e_block(), H.B, beta, H.disp[sd].dev, H.stream);
        n += 2;
    }
    // the SIBC walls after the mu-side ADE (fit_td.py:903-914)
    if (sibc) {
        launch_sibc_update<T>(F, H.e_block(), H.B, beta, H.sibc.dev, H.stream);
        n += 2;
    }
    StencilArgs<T> sa = stencil_args<T>(H);
    for (int q = 0; q < sa.nfaces; ++q) {
        launch_cpml_pass<T>(sa, q, sd, H.stream);
        ++n;
    }
    return n;
}

// Fork: the DTBC convolutions of this step start on the side stream as soon
// as the previous step's port update has written its history; join: the
// port update waits for them.  Returns the launches issued.
int fork_dtbc_conv(Handle& H, const PortsArgs& pa) {
    if (H.modal.empty() || !H.any_dtbc()) return 0;
    ck(cudaEventRecord(H.ev_fork, H.stream), "fork record");
    ck(cudaStreamWaitEvent(H.side, H.ev_fork, 0), "fork wait");
    launch_dtbc_conv(pa, H.d_modal.as<ModalDev>(), (int)H.modal.size(),
                     (int)((H.cap + kConvChunk - 1) / kConvChunk), H.side);
    ck(cudaEventRecord(H.ev_join, H.side), "join record");
    return 1;
}

void join_dtbc_conv(Handle& H) {
    if (H.modal.empty() || !H.any_dtbc()) return;
    ck(cudaStreamWaitEvent(H.stream, H.ev_join, 0), "join wait");
}

// Fused step: one launch for E and H from the current buffer set into the
// other, then the ports on the new E (with the old H, which the two-pass
// order shows them), the H fix-up next to port edges, the monitors on the
// new fields; the buffer sets swap.
template <typename T>
int enqueue_step_fused(Handle& H) {
    int n = 0;
    PortsArgs pa = ports_args(H);
    StencilArgs<T> sa = stencil_args<T>(H);
    n += fork_dtbc_conv(H, pa);
    // ADE (slab step only): the pole histories take the fields before the
    // step, which the current buffer set still holds
    for (int sd = 0; sd < 2; ++sd) {
        if (!H.disp[sd].present()) continue;
        launch_disp_save<T>((sd == 0 ? H.Ec() : H.Hc()).as<T>(), H.e_block(), H.B, H.disp[sd].dev, H.stream);
        ++n;
    }
    n += launch_fused<T>(H, sa);
    T* e_new = H.En().as<T>();
    T* h_new = H.Hn().as<T>();
    if (H.disp[0].present()) {
        // E-side ADE after the curl update and the CPML (which never share
        // an entry with it, disp_clear_of_cpml), before the ports
        launch_disp_update<T>(e_new, H.e_block(), H.B, H.bE.as<T>(), H.disp[0].dev, H.stream);
        n += 2;
    }
    for (auto& pw : H.pws) {
        launch_plane_wave<T>(e_new, H.e_block(), H.B, pw->dev, 0, H.step.as<long long>(), H.stream);
        ++n;
    }
    if (!H.modal.empty()) {
        join_dtbc_conv(H);
        launch_modal<T>(e_new, H.Hc().as<T>(), pa, H.d_modal.as<ModalDev>(), (int)H.modal.size(), H.modal_chunks,
                        H.stream);
        ++n;
    }
    if (!H.lumped.empty()) {
        launch_lumped<T>(e_new, pa, H.d_lumped.as<LumpedDev>(), (int)H.lumped.size(), H.stream);
        ++n;
    }
    if (is_tile_variant(H.fused_variant)) {
        const int nh = launch_tile_cpml_H<T>(sa, H.stream);
        if (nh < 0) fail(FITB_ERR_STATE, "the tile step does not take this grid / CPML layout");
        n += nh;
    }
    if (H.n_fix > 0) {
        launch_fix_H<T>(sa, H.fix_cells.as<int4>(), H.n_fix, H.stream);
        ++n;
    }
    if (H.disp[1].present()) {
        launch_disp_update<T>(h_new, H.e_block(), H.B, H.bH.as<T>(), H.disp[1].dev, H.stream);
        n += 2;
    }
    for (auto& pw : H.pws) {
        launch_plane_wave<T>(h_new, H.e_block(), H.B, pw->dev, 1, H.step.as<long long>(), H.stream);
        ++n;
    }
    if (!H.dft.empty()) {
        launch_dft_stage_all<T>(e_new, h_new, H.e_block(), H.e_block(), H.g, H.B, H.d_dft.as<DftDev>(),
                                (int)H.dft.size(), H.dft_stage_blocks, H.step.as<long long>(), H.stream);
        launch_dft_flush_all(H.B, H.d_dft.as<DftDev>(), (int)H.dft.size(), H.dft_flush_blocks, H.dft_flush_smem,
                             H.step.as<long long>(), H.ticket.as<unsigned>(), H.stream);
        n += 2;
    } else {
        launch_advance(H.step.as<long long>(), H.stream);
        ++n;
    }
    H.cur ^= 1;
    return n;
}

template <typename T>
int enqueue_step(Handle& H) {
    if (H.stencil_mode == kModeFused) return enqueue_step_fused<T>(H);
    // in-place kernels below
    int n = 0;
    PortsArgs pa = ports_args(H);
    n += fork_dtbc_conv(H, pa);
    for (int sd = 0; sd < 2; ++sd) {
        if (!H.disp[sd].present()) continue;
        launch_disp_save<T>((sd == 0 ? H.Ec() : H.Hc()).as<T>(), H.e_block(), H.B, H.disp[sd].dev, H.stream);
        ++n;
    }
    if (H.sibc.present()) {
        launch_sibc_save<T>(H.Hc().as<T>(), H.e_block(), H.B, H.sibc.dev, H.stream);
        ++n;
    }
    launch_half<T>(H, 0);
    ++n;
    n += disp_complete<T>(H, 0);
    for (auto& pw : H.pws) {
        launch_plane_wave<T>(H.Ec().as<T>(), H.e_block(), H.B, pw->dev, 0, H.step.as<long long>(), H.stream);
        ++n;
    }
    if (!H.modal.empty()) {
        join_dtbc_conv(H);
        launch_modal<T>(H.Ec().as<T>(), H.Hc().as<T>(), pa, H.d_modal.as<ModalDev>(), (int)H.modal.size(),
                        H.modal_chunks, H.stream);
        ++n;
    }
    if (!H.band.empty()) {
        launch_band<T>(H.Ec().as<T>(), H.Hc().as<T>(), pa, H.d_band.as<BandDev>(), (int)H.band.size(),
                       (int)((H.cap + kConvChunk - 1) / kConvChunk), H.stream);
        n += 2;
    }
    if (!H.lumped.empty()) {
        launch_lumped<T>(H.Ec().as<T>(), pa, H.d_lumped.as<LumpedDev>(), (int)H.lumped.size(), H.stream);
        ++n;
    }
    launch_half<T>(H, 1);
    ++n;
    n += disp_complete<T>(H, 1);
    for (auto& pw : H.pws) {
        launch_plane_wave<T>(H.Hc().as<T>(), H.e_block(), H.B, pw->dev, 1, H.step.as<long long>(), H.stream);
        ++n;
    }
    if (!H.dft.empty()) {
        // stage + flush of all monitors; the flush launch advances the step
        launch_dft_stage_all<T>(H.Ec().as<T>(), H.Hc().as<T>(), H.e_block(), H.e_block(), H.g, H.B,
                                H.d_dft.as<DftDev>(), (int)H.dft.size(), H.dft_stage_blocks, H.step.as<long long>(),
                                H.stream);
        launch_dft_flush_all(H.B, H.d_dft.as<DftDev>(), (int)H.dft.size(), H.dft_flush_blocks, H.dft_flush_smem,
                             H.step.as<long long>(), H.ticket.as<unsigned>(), H.stream);
        n += 2;
    } else {
        launch_advance(H.step.as<long long>(), H.stream);
        ++n;
    }
    return n;
}

int enqueue_step_any(Handle& H) { return H.prec == 4 ? enqueue_step<float>(H) : enqueue_step<double>(H); }

// Captures nsteps steps starting from the current buffer set; the host-side
// buffer set index is restored (the graph has not run yet).
cudaGraphExec_t capture(Handle& H, int nsteps, int* launches_per) {
    cudaGraph_t graph = nullptr;
    const int cur0 = H.cur;
    struct Restore {
        Handle& H;
        int c;
        ~Restore() { H.cur = c; }
    } restore{H, cur0};
    ck(cudaStreamBeginCapture(H.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int per = 0;
    try {
        for (int s = 0; s < nsteps; ++s) per = enqueue_step_any(H);
    } catch (...) {
        cudaStreamEndCapture(H.stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    ck(cudaStreamEndCapture(H.stream, &graph), "end capture");
    cudaGraphExec_t exec = nullptr;
    cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    ck(err, "graph instantiate");
    *launches_per = per;
    return exec;
}

// Reads (and clears) the device status word of the pipelined stencil
// kernels; a non-zero value means a bounded shared-memory pipeline wait
// expired and the step's results are not valid.
// the stencil forms whose copy pipelines record a status word
bool has_device_status(const Handle& H) {
    return H.stencil_mode == kModeBulk || (H.stencil_mode == kModeFused && H.fused_variant >= kFusedTileBase);
}

// error out on a nonzero status word `st` (read after the step), resetting it
void raise_device_status(Handle& H, int st) {
    if (st != 0) {
        ck(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream), "status reset");
        fail(FITB_ERR_CUDA, "a bounded wait in the %s copy pipeline expired (status %d)",
             st == kStatusWaitTimeoutE ? "E-update" : (st == kStatusWaitTimeoutH ? "H-update" : "tile-step"), st);
    }
}

void check_device_status(Handle& H) {
    if (!has_device_status(H)) return;
    int st = 0;
    ck(cudaMemcpyAsync(&st, H.status.p, sizeof(int), cudaMemcpyDeviceToHost, H.stream), "status D2H");
    ck(cudaStreamSynchronize(H.stream), "status sync");
    raise_device_status(H, st);
}

void check_ready(Handle& H) {
    if (!H.coeffs_set) fail(FITB_ERR_STATE, "coefficients not set (call fitb_set_coeffs first)");
}

void check_dtbc_tables(Handle& H, long long last_step) {
    // Chain step n uses the table of length n0 * 2^t >= n + 1.
    for (size_t p = 0; p < H.modal.size(); ++p) {
        auto& mp = *H.modal[p];
        long long tlen = mp.dev.n0;
        int t = 0;
        while (tlen < last_step + 1) {
            tlen *= 2;
            ++t;
        }
        for (int m = 0; m < mp.n_modes; ++m) {
            if (!mp.dev.is_dtbc[m]) continue;
            if (mp.n_tables_mode[m] <= t)
                fail(FITB_ERR_STATE,
                     "modal port %zu mode %d: DTBC kernel table of length %lld missing for step %lld "
                     "(call fitb_set_dtbc_kernel)",
                     p, m, tlen, last_step);
        }
    }
    for (size_t q = 0; q < H.band.size(); ++q) {
        const auto& bp = *H.band[q];
        long long tlen = bp.dev.n0;
        int t = 0;
        while (tlen < last_step + 1) {
            tlen *= 2;
            ++t;
        }
        if (bp.n_out <= t || (bp.n_in > 0 && bp.n_in <= t))
            fail(FITB_ERR_STATE,
                 "band port %zu: DTBC kernel table of length %lld missing for step %lld (call fitb_set_band_kernel)",
                 q, tlen, last_step);
    }
}

void run_steps(Handle& H, long long nsteps) {
    check_ready(H);
    if (nsteps < 0) fail(FITB_ERR_ARG, "n_steps must be >= 0");
    if (nsteps > 0) check_dtbc_tables(H, H.steps_done + nsteps - 1);
    ensure_capacity(H, H.steps_done + nsteps);
    refresh_port_tables(H);
    sync_dead_units(H);
    int per = 0;
    if (!H.graphs_valid) {
        // a capture that failed part-way left the graphs it had finished:
        // free them before capturing again
        invalidate_graphs(H);
        // graphs for each starting buffer set (one set for in-place kernels)
        const int nsets = H.stencil_mode == kModeFused ? 2 : 1;
        const int cur0 = H.cur;
        int p1 = 0, pc = 0;
        for (int q = 0; q < nsets; ++q) {
            H.cur = q;
            H.graph_one[q] = capture(H, 1, &p1);
            H.graph_chunk[q] = capture(H, H.chunk, &pc);
        }
        H.cur = cur0;
        H.graphs_valid = true;
        H.launches_per_step = p1;
    }
    per = H.launches_per_step;
    if (nsteps == 0) return;
    long long left = nsteps;
    const bool swaps = H.stencil_mode == kModeFused;
    while (left >= H.chunk) {
        ck(cudaGraphLaunch(H.graph_chunk[H.cur], H.stream), "graph launch");
        if (swaps && (H.chunk & 1)) H.cur ^= 1;
        left -= H.chunk;
    }
    while (left > 0) {
        ck(cudaGraphLaunch(H.graph_one[H.cur], H.stream), "graph launch");
        if (swaps) H.cur ^= 1;
        --left;
    }
    H.launches += (long long)per * nsteps;
    H.steps_done += nsteps;
}

template <typename T>
void energy_impl(Handle& H, int b, double* out) {
    launch_energy<T>(H.Ec().as<T>(), H.Hc().as<T>(), H.meps.as<T>(), H.mmu.as<T>(), H.g, b, H.e_block(),
                     H.energy_partials.as<double>(), H.energy_blocks, H.energy_out.as<double>(), H.stream);
    H.launches += 2;
    ck(cudaGetLastError(), "energy");
    ck(cudaMemcpyAsync(out, H.energy_out.p, sizeof(double), cudaMemcpyDeviceToHost, H.stream), "energy D2H");
    ck(cudaStreamSynchronize(H.stream), "energy sync");
    check_device_status(H);
}

long long dft_recorded_upto(long long x, int stride) { return x < 0 ? 0 : x / stride + 1; }

// Flush the partially filled slot block of every monitor and restart the
// slot count at the next step.
void dft_flush_pending(Handle& H) {
    for (auto& mp : H.dft) {
        DftHost& m = *mp;
        long long cnt = dft_recorded_upto(H.steps_done - 1, m.dev.stride) -
                        dft_recorded_upto(m.base_host - 1, m.dev.stride);
        int pending = (int)(cnt % m.dev.K);
        if (pending > 0) {
            launch_dft_flush_forced(H.B, m.dev, pending, H.stream);
            H.launches++;
            ck(cudaGetLastError(), "dft flush");
        }
        m.base_host = H.steps_done;
        ck(cudaMemcpyAsync(m.base.p, &m.base_host, sizeof(long long), cudaMemcpyHostToDevice, H.stream),
           "dft base");
        ck(cudaStreamSynchronize(H.stream), "dft flush sync");
    }
}

int face_axis(int face) { return face / 2; }

// Reference psi shape of auxiliary q (0..3 = E1,E2,H1,H2) on a face axis.
void psi_ref_shape(const Geom& g, int axis, int n, int q, int& a, int& b, int& c) {
    static const int comps[3][4] = {{1, 2, 4, 5}, {0, 2, 3, 5}, {0, 1, 3, 4}};
    comp_shape(g, comps[axis][q], a, b, c);
    if (axis == 0) a = n;
    if (axis == 1) b = n;
    if (axis == 2) c = n;
}

template <typename T>
void add_cpml_impl(Handle& H, int face, int n_pml, const double* bt, const double* ct, const double* ckt,
                   const uint8_t* const air_in[4]) {
    auto f = std::make_unique<FaceHost>();
    f->face = face;
    const int axis = face_axis(face), side = face % 2;
    const int N = axis == 0 ? H.g.nx : (axis == 1 ? H.g.ny : H.g.nz);
    if (n_pml < 1 || n_pml > N) fail(FITB_ERR_ARG, "n_pml %d out of range [1, %d]", n_pml, N);
    FaceDev& d = f->dev;
    d.axis = axis;
    d.n = n_pml;
    d.lo = side == 0 ? 0 : N - n_pml;
    d.dI = axis == 0 ? n_pml : H.g.nx + 1;
    d.dJ = axis == 1 ? n_pml : H.g.ny + 1;
    d.dK = axis == 2 ? n_pml : H.g.nz + 1;
    // rows padded to 16 entries: whole rows stay 16-byte aligned for the
    // psi (field dtype) and air (byte) tensor copies of the tile step
    d.pk = (int)round_up(d.dK, 16);
    d.slab = (long long)d.dI * d.dJ * d.pk;
    f->psi.alloc((size_t)H.B * 4 * d.slab * sizeof(T));
    if (H.stencil_mode == kModeFused) f->psi2.alloc((size_t)H.B * 4 * d.slab * sizeof(T));
    std::vector<uint8_t> air((size_t)(4 * d.slab), 0);
    for (int q = 0; q < 4; ++q) {
        int ra, rb, rc;
        psi_ref_shape(H.g, axis, n_pml, q, ra, rb, rc);
        for (int x = 0; x < ra; ++x)
            for (int y = 0; y < rb; ++y)
                for (int z = 0; z < rc; ++z) {
                    long long src = ((long long)x * rb + y) * rc + z;
                    long long dst = (long long)q * d.slab + ((long long)x * d.dJ + y) * d.pk + z;
                    air[(size_t)dst] = air_in[q] ? (air_in[q][src] ? 1 : 0) : 1;
                    if (!air[(size_t)dst]) f->pec = true;
                }
    }
    upload(f->air, air);
    std::vector<T> bcc((size_t)(3 * n_pml));
    for (int l = 0; l < n_pml; ++l) {
        bcc[(size_t)l] = (T)bt[l];
        bcc[(size_t)(n_pml + l)] = (T)ct[l];
        bcc[(size_t)(2 * n_pml + l)] = (T)ckt[l];
    }
    upload(f->bcc, bcc);
    d.psi = f->psi.p;
    d.psi_next = f->psi2.p;
    d.air = f->air.as<unsigned char>();
    d.bcc = f->bcc.p;
    H.faces.push_back(std::move(f));
}

// ---- state serialisation ----------------------------------------------
struct Writer {
    std::vector<char>* out = nullptr;  // sizing pass when null
    size_t n = 0;
    void put(const void* p, size_t bytes) {
        if (out) out->insert(out->end(), (const char*)p, (const char*)p + bytes);
        n += bytes;
    }
    template <typename U>
    void pod(const U& v) {
        put(&v, sizeof(U));
    }
};

void dev_get(Writer& w, const void* dptr, size_t bytes) {
    if (!w.out) {
        w.n += bytes;
        return;
    }
    size_t at = w.out->size();
    w.out->resize(at + bytes);
    if (bytes) ck(cudaMemcpy(w.out->data() + at, dptr, bytes, cudaMemcpyDeviceToHost), "state D2H");
    w.n += bytes;
}

template <typename T>
void write_state(Handle& H, Writer& w) {
    const unsigned long long magic = 0x46495442'32303031ULL;  // "FITB2001"
    w.pod(magic);
    w.pod((int)H.prec);
    w.pod((int)H.B);
    w.pod(H.g.nx);
    w.pod(H.g.ny);
    w.pod(H.g.nz);
    w.pod(H.steps_done);
    // fields in the reference flat layout
    for (int b = 0; b < H.B; ++b) {
        std::vector<T> ev, hv;
        if (w.out) {
            ev.resize((size_t)H.nE());
            hv.resize((size_t)H.nH());
            unpack3<T>(H, H.Ec().as<T>() + (long long)b * H.e_block(), ev.data(), 0);
            unpack3<T>(H, H.Hc().as<T>() + (long long)b * H.e_block(), hv.data(), 3);
        }
        if (w.out) {
            w.put(ev.data(), ev.size() * sizeof(T));
            w.put(hv.data(), hv.size() * sizeof(T));
        } else {
            w.n += (size_t)(H.nE() + H.nH()) * sizeof(T);
        }
    }
    for (auto& f : H.faces) {
        const DevBuf& ps = H.cur ? f->psi2 : f->psi;
        dev_get(w, ps.p, ps.bytes);
    }
    for (auto& dp : H.disp) dev_get(w, dp.d_J.p, dp.d_J.bytes);
    dev_get(w, H.sibc.d_u.p, H.sibc.d_u.bytes);
    for (auto& bp : H.band) {
        dev_get(w, bp->st.p, bp->st.bytes);
        dev_get(w, bp->x1prev.p, bp->x1prev.bytes);
        const size_t row = (size_t)bp->p * sizeof(double);
        for (int b = 0; b < H.B; ++b)
            for (DevBuf* hb : {&bp->whist, &bp->shist})
                dev_get(w, hb->as<char>() + (size_t)b * H.cap * row, (size_t)H.steps_done * row);
    }
    for (auto& lp : H.lumped) dev_get(w, lp->st.p, lp->st.bytes);
    for (auto& mp : H.modal) {
        dev_get(w, mp->st.p, mp->st.bytes);
        dev_get(w, mp->comp_state.p, mp->comp_state.bytes);
        // histories up to the completed step count, per (b, mode)
        int M = mp->n_modes;
        for (int b = 0; b < H.B; ++b)
            for (int m = 0; m < M; ++m) {
                size_t off = (((size_t)b * M + m) * (size_t)H.cap) * sizeof(double);
                dev_get(w, mp->whist.as<char>() + off, (size_t)H.steps_done * sizeof(double));
                dev_get(w, mp->shist.as<char>() + off, (size_t)H.steps_done * sizeof(double));
            }
    }
    for (auto& m : H.dft) {
        dev_get(w, m->bins.p, m->bins.bytes);
        dev_get(w, m->cmp.p, m->cmp.bytes);
    }
    dev_get(w, H.absmax.p, H.absmax.bytes);
}

struct Reader {
    const char* p;
    size_t left;
    void get(void* dst, size_t bytes) {
        if (bytes > left) fail(FITB_ERR_ARG, "state buffer too short");
        memcpy(dst, p, bytes);
        p += bytes;
        left -= bytes;
    }
    void dev(void* dptr, size_t bytes) {
        if (bytes > left) fail(FITB_ERR_ARG, "state buffer too short");
        if (bytes) ck(cudaMemcpy(dptr, p, bytes, cudaMemcpyHostToDevice), "state H2D");
        p += bytes;
        left -= bytes;
    }
    template <typename U>
    U pod() {
        U v;
        get(&v, sizeof(U));
        return v;
    }
};

template <typename T>
void read_state(Handle& H, Reader& r) {
    const unsigned long long magic = 0x46495442'32303031ULL;
    if (r.pod<unsigned long long>() != magic) fail(FITB_ERR_ARG, "not a fitb200 state buffer");
    int prec = r.pod<int>(), B = r.pod<int>(), nx = r.pod<int>(), ny = r.pod<int>(), nz = r.pod<int>();
    if (prec != H.prec || B != H.B || nx != H.g.nx || ny != H.g.ny || nz != H.g.nz)
        fail(FITB_ERR_ARG, "state buffer was written by a differently configured handle");
    long long steps = r.pod<long long>();
    ck(cudaStreamSynchronize(H.stream), "state import sync");
    ensure_capacity(H, steps + 1);
    for (int b = 0; b < H.B; ++b) {
        std::vector<T> ev((size_t)H.nE()), hv((size_t)H.nH());
        r.get(ev.data(), ev.size() * sizeof(T));
        r.get(hv.data(), hv.size() * sizeof(T));
        pack3<T>(H, ev.data(), H.Ec().as<T>() + (long long)b * H.e_block(), 0);
        pack3<T>(H, hv.data(), H.Hc().as<T>() + (long long)b * H.e_block(), 3);
    }
    for (auto& f : H.faces) {
        DevBuf& ps = H.cur ? f->psi2 : f->psi;
        r.dev(ps.p, ps.bytes);
    }
    for (auto& dp : H.disp) r.dev(dp.d_J.p, dp.d_J.bytes);
    r.dev(H.sibc.d_u.p, H.sibc.d_u.bytes);
    for (auto& bp : H.band) {
        r.dev(bp->st.p, bp->st.bytes);
        r.dev(bp->x1prev.p, bp->x1prev.bytes);
        const size_t row = (size_t)bp->p * sizeof(double);
        for (int b = 0; b < H.B; ++b)
            for (DevBuf* hb : {&bp->whist, &bp->shist})
                r.dev(hb->as<char>() + (size_t)b * H.cap * row, (size_t)steps * row);
    }
    for (auto& lp : H.lumped) r.dev(lp->st.p, lp->st.bytes);
    for (auto& mp : H.modal) {
        r.dev(mp->st.p, mp->st.bytes);
        r.dev(mp->comp_state.p, mp->comp_state.bytes);
        int M = mp->n_modes;
        ck(cudaMemset(mp->whist.p, 0, mp->whist.bytes), "clear history");
        ck(cudaMemset(mp->shist.p, 0, mp->shist.bytes), "clear history");
        for (int b = 0; b < H.B; ++b)
            for (int m = 0; m < M; ++m) {
                size_t off = (((size_t)b * M + m) * (size_t)H.cap) * sizeof(double);
                r.dev(mp->whist.as<char>() + off, (size_t)steps * sizeof(double));
                r.dev(mp->shist.as<char>() + off, (size_t)steps * sizeof(double));
            }
    }
    for (auto& m : H.dft) {
        r.dev(m->bins.p, m->bins.bytes);
        r.dev(m->cmp.p, m->cmp.bytes);
    }
    r.dev(H.absmax.p, H.absmax.bytes);
    H.steps_done = steps;
    ck(cudaMemcpy(H.step.p, &steps, sizeof(long long), cudaMemcpyHostToDevice), "step counter");
    for (auto& m : H.dft) {
        m->base_host = steps;
        ck(cudaMemcpy(m->base.p, &steps, sizeof(long long), cudaMemcpyHostToDevice), "dft base");
    }
    legacy_sync("state import copy sync");
}

}  // namespace
}  // namespace fitb

// ===========================================================================
// C ABI
// ===========================================================================
using fitb::Handle;

#define FITB_TRY try {
#define FITB_CATCH                                                   \
    }                                                                \
    catch (const fitb::Error& ex) {                                  \
        fitb::g_last_error = ex.what();                              \
        return ex.code;                                              \
    }                                                                \
    catch (const std::bad_alloc&) {                                  \
        fitb::g_last_error = "host allocation failed";               \
        return FITB_ERR_NOMEM;                                       \
    }                                                                \
    catch (const std::exception& ex) {                               \
        fitb::g_last_error = ex.what();                              \
        return FITB_ERR_STATE;                                       \
    }                                                                \
    return FITB_OK;

static Handle& H_of(fitb_handle* h) {
    if (!h) fail(FITB_ERR_ARG, "null handle");
    ck(cudaSetDevice(h->impl.desc.device), "cudaSetDevice");
    return h->impl;
}

extern "C" {

int fitb_abi_version(void) { return FITB_ABI_VERSION; }

int fitb_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return FITB_ERR_ARG;
    snprintf(buf, len, "%s", fitb::g_last_error.c_str());
    return FITB_OK;
}

int fitb_create(const fitb_desc* desc, fitb_handle** out) {
    FITB_TRY
    if (!desc || !out) fail(FITB_ERR_ARG, "null argument");
    *out = nullptr;
    if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1) fail(FITB_ERR_ARG, "grid must have >= 1 cell per axis");
    if (desc->batch < 1) fail(FITB_ERR_ARG, "batch must be >= 1");
    if (desc->precision != 4 && desc->precision != 8) fail(FITB_ERR_ARG, "precision must be 4 or 8");
    if (!(desc->dt > 0.0)) fail(FITB_ERR_ARG, "dt must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        fail(FITB_ERR_NODEV, "no CUDA device available");
    }
    if (desc->device < 0 || desc->device >= ndev) fail(FITB_ERR_ARG, "device %d out of range", desc->device);
    ck(cudaSetDevice(desc->device), "cudaSetDevice");
    auto owner = std::make_unique<fitb_handle>();
    Handle& H = owner->impl;
    H.desc = *desc;
    H.prec = desc->precision;
    H.esz = (size_t)desc->precision;
    H.B = desc->batch;
    H.dt = desc->dt;
    fitb::Geom& g = H.g;
    g.nx = desc->nx;
    g.ny = desc->ny;
    g.nz = desc->nz;
    g.njp = g.ny + 2;
    g.nkp = (int)fitb::round_up(g.nz + 2, 8);
    g.sj = g.nkp;
    g.si = (long long)g.njp * g.nkp;
    g.vol = (long long)(g.nx + 4) * g.si + (long long)fitb::kTailRows * g.sj;
    ck(cudaStreamCreateWithFlags(&H.stream, cudaStreamNonBlocking), "stream");
    ck(cudaStreamCreateWithFlags(&H.side, cudaStreamNonBlocking), "stream");
    ck(cudaEventCreateWithFlags(&H.ev_fork, cudaEventDisableTiming), "event");
    ck(cudaEventCreateWithFlags(&H.ev_join, cudaEventDisableTiming), "event");
    ck(cudaEventCreateWithFlags(&H.ev_sfork, cudaEventDisableTiming), "event");
    for (auto& t : H.tickets) ck(cudaEventCreateWithFlags(&t, cudaEventDisableTiming), "event");
    for (int q = 1; q < fitb::kSlabLists; ++q) {
        ck(cudaStreamCreateWithFlags(&H.slab_side[q], cudaStreamNonBlocking), "stream");
        ck(cudaEventCreateWithFlags(&H.ev_sjoin[q], cudaEventDisableTiming), "event");
    }
    const size_t blk = (size_t)H.e_block() * H.esz;
    H.e.alloc(blk * H.B);
    H.h.alloc(blk * H.B);
    H.aE.alloc(blk);
    H.bE.alloc(blk);
    H.aH.alloc(blk);
    H.bH.alloc(blk);
    H.meps.alloc(blk);
    H.mmu.alloc(blk);
    H.staging.alloc((size_t)std::max(H.nE(), H.nH()) * H.esz, false);
    H.step.alloc(sizeof(long long));
    H.absmax.alloc(sizeof(double) * H.B);
    H.energy_partials.alloc(sizeof(double) * H.energy_blocks);
    H.energy_out.alloc(sizeof(double));
    H.status.alloc(sizeof(int));
    H.ticket.alloc(sizeof(unsigned));
    {
        // FITB_STENCIL selects the stencil kernels: "stream" (default),
        // "fused" (E and H in one pass over ping-pong buffers;
        // FITB_FUSED_VARIANT picks the kernel form), "vec" (vectorised planes;
        // FITB_VEC_VARIANT picks the vector width and register cap), "bulk"
        // (cp.async.bulk pipeline, one field set) or "simple".
        const char* mode = getenv("FITB_STENCIL");
        const std::string m = mode ? mode : "stream";
        H.stencil_mode = fitb::kModeSimple;
        if (H.B == 1 && m == "bulk") {
            int sms = 148;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, desc->device);
            H.plan = H.prec == 4 ? fitb::plan_bulk<float>(g, sms) : fitb::plan_bulk<double>(g, sms);
            if (H.plan.stages >= 3) {
                ck(H.prec == 4 ? fitb::prepare_bulk<float>(H.plan) : fitb::prepare_bulk<double>(H.plan),
                   "bulk stencil smem attribute");
                H.stencil_mode = fitb::kModeBulk;
            }
        } else if (m == "fused") {
            const char* t = getenv("FITB_FUSED_VARIANT");
            H.fused_variant = t ? std::max(0, std::min(fitb::kFusedSlabBase + fitb::kSlabVariants - 1, atoi(t))) : 2;
            if (H.fused_variant == 1 && H.prec == 8) H.fused_variant = 0;
            if (!fitb::fused_variant_ok(H.prec, H.fused_variant) ||
                (fitb::is_slab_variant(H.fused_variant) &&
                 H.B % fitb::slab_nb_of(H.fused_variant - fitb::kFusedSlabBase) != 0))
                H.fused_variant = 2;
            ck(fitb::prepare_fused_any(H.prec, H.fused_variant), "fused step smem attribute");
            H.e2.alloc(blk * H.B);
            H.h2.alloc(blk * H.B);
            H.stencil_mode = fitb::kModeFused;
        } else if (m == "vec" && H.B <= 8 && fitb::stream_batch_supported(H.B)) {
            const char* v = getenv("FITB_VEC_VARIANT");
            H.vec_variant = v ? std::max(0, std::min(3, atoi(v))) : 0;
            H.stencil_mode = fitb::kModeVec;
        } else if (fitb::stream_batch_supported(H.B) && m != "simple") {
            H.stencil_mode = fitb::kModeStream;
        }
        fitb::plan_stencil(H);
    }
    *out = owner.release();
    FITB_CATCH
}

int fitb_destroy(fitb_handle* h) {
    FITB_TRY
    if (!h) return FITB_OK;
    cudaSetDevice(h->impl.desc.device);
    cudaStreamSynchronize(h->impl.stream);
    delete h;
    FITB_CATCH
}

int fitb_launch_count(const fitb_handle* h, int64_t* out) {
    FITB_TRY
    if (!h || !out) fail(FITB_ERR_ARG, "null argument");
    *out = h->impl.launches;
    FITB_CATCH
}

int fitb_set_coeffs(fitb_handle* h, const double* alpha_e, const double* beta_e, const double* alpha_h,
                    const double* beta_h, const double* m_eps, const double* m_mu) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!alpha_e || !beta_e || !alpha_h || !beta_h) fail(FITB_ERR_ARG, "null coefficient array");
    const long long nE = H.nE(), nH = H.nH();
    auto put = [&](fitb::DevBuf& dst, const double* src, long long n, int c0) {
        if (H.prec == 4) {
            std::vector<float> v = fitb::cast_vec<float>(src, n);
            fitb::pack3<float>(H, v.data(), dst.as<float>(), c0);
        } else {
            fitb::pack3<double>(H, src, dst.as<double>(), c0);
        }
    };
    put(H.aE, alpha_e, nE, 0);
    put(H.bE, beta_e, nE, 0);
    put(H.aH, alpha_h, nH, 3);
    put(H.bH, beta_h, nH, 3);
    if (m_eps) put(H.meps, m_eps, nE, 0);
    if (m_mu) put(H.mmu, m_mu, nH, 3);
    fitb::comp_max(H, alpha_e, 0, H.coef_max[0]);
    fitb::comp_max(H, beta_e, 0, H.coef_max[1]);
    fitb::comp_max(H, alpha_h, 3, H.coef_max[2]);
    fitb::comp_max(H, beta_h, 3, H.coef_max[3]);
    H.coeffs_set = true;
    fitb::compact_coeffs(H);
    H.port_tables_dirty = true;  // the slab step's dead-unit plan reads the coefficients
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_build_materials(fitb_handle* h, const double* dx, const double* dy, const double* dz, const int32_t* mat_id,
                         int32_t n_mat, const double* eps_r, int64_t n_cat1, const int64_t* cat1_idx,
                         const double* cat1_eps, int64_t n_pec, const int64_t* pec_idx) {
    FITB_TRY
    Handle& H = H_of(h);
    const fitb::Geom& g = H.g;
    if (!dx || !dy || !dz || !mat_id || !eps_r || n_mat < 1) fail(FITB_ERR_ARG, "null array or no materials");
    if (n_cat1 < 0 || n_pec < 0 || (n_cat1 > 0 && (!cat1_idx || !cat1_eps)) || (n_pec > 0 && !pec_idx))
        fail(FITB_ERR_ARG, "cat-1 / PEC lists");
    const long long cells = (long long)g.nx * g.ny * g.nz;
    for (long long q = 0; q < cells; ++q)
        if (mat_id[q] < 0 || mat_id[q] >= n_mat) fail(FITB_ERR_ARG, "material id %d of cell %lld", mat_id[q], q);
    const long long nE = H.nE();
    for (long long q = 0; q < n_cat1; ++q)
        if (cat1_idx[q] < 0 || cat1_idx[q] >= nE) fail(FITB_ERR_ARG, "cat-1 edge %lld", (long long)cat1_idx[q]);
    for (long long q = 0; q < n_pec; ++q)
        if (pec_idx[q] < 0 || pec_idx[q] >= nE) fail(FITB_ERR_ARG, "PEC edge %lld", (long long)pec_idx[q]);
    ck(cudaStreamSynchronize(H.stream), "sync");
    fitb::DevBuf ddx, ddy, ddz, dmat, deps, dci, dce, dpi, dmax;
    fitb::upload(ddx, std::vector<double>(dx, dx + g.nx));
    fitb::upload(ddy, std::vector<double>(dy, dy + g.ny));
    fitb::upload(ddz, std::vector<double>(dz, dz + g.nz));
    fitb::upload(dmat, std::vector<int>(mat_id, mat_id + cells));
    fitb::upload(deps, std::vector<double>(eps_r, eps_r + n_mat));
    fitb::upload(dci, std::vector<long long>(cat1_idx, cat1_idx + n_cat1 + (n_cat1 == 0)));
    fitb::upload(dce, std::vector<double>(cat1_eps, cat1_eps + n_cat1 + (n_cat1 == 0)));
    fitb::upload(dpi, std::vector<long long>(pec_idx, pec_idx + n_pec + (n_pec == 0)));
    dmax.alloc(12 * sizeof(double));
    if (H.prec == 4)
        fitb::launch_setup_materials<float>(g, ddx.as<double>(), ddy.as<double>(), ddz.as<double>(), dmat.as<int>(),
                                            deps.as<double>(), H.dt, n_cat1, dci.as<long long>(), dce.as<double>(),
                                            n_pec, dpi.as<long long>(), H.aE.as<float>(), H.bE.as<float>(),
                                            H.aH.as<float>(), H.bH.as<float>(), H.meps.as<float>(),
                                            H.mmu.as<float>(), dmax.as<double>(), H.stream);
    else
        fitb::launch_setup_materials<double>(g, ddx.as<double>(), ddy.as<double>(), ddz.as<double>(),
                                             dmat.as<int>(), deps.as<double>(), H.dt, n_cat1, dci.as<long long>(),
                                             dce.as<double>(), n_pec, dpi.as<long long>(), H.aE.as<double>(),
                                             H.bE.as<double>(), H.aH.as<double>(), H.bH.as<double>(),
                                             H.meps.as<double>(), H.mmu.as<double>(), dmax.as<double>(), H.stream);
    ck(cudaGetLastError(), "material setup launch");
    double mx[12];
    ck(cudaMemcpyAsync(mx, dmax.p, sizeof(mx), cudaMemcpyDeviceToHost, H.stream), "coefficient max D2H");
    ck(cudaStreamSynchronize(H.stream), "material setup sync");
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) H.coef_max[a][c] = mx[3 * a + c];
    H.launches += 5;
    H.coeffs_set = true;
    fitb::compact_coeffs(H);
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_spectral_dt(fitb_handle* h, double safety, int32_t max_iter, double tol, double* lambda_max, double* dt,
                     int32_t* iterations) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!lambda_max || !dt || max_iter < 1 || !(tol > 0.0) || !(safety > 0.0)) fail(FITB_ERR_ARG, "bad argument");
    if (!H.coeffs_set) fail(FITB_ERR_STATE, "coefficients (with M_eps and M_mu) must be set first");
    ck(cudaStreamSynchronize(H.stream), "sync");
    double lam = 0.0;
    int its = 0;
    const int rc = H.prec == 4 ? fitb::spectral_lambda<float>(H.g, H.meps.as<float>(), H.mmu.as<float>(),
                                                              H.bE.as<float>(), max_iter, tol, &lam, &its, H.stream)
                               : fitb::spectral_lambda<double>(H.g, H.meps.as<double>(), H.mmu.as<double>(),
                                                               H.bE.as<double>(), max_iter, tol, &lam, &its, H.stream);
    if (rc == -1) fail(FITB_ERR_CUDA, "spectral dt: device memory for the Lanczos vectors");
    if (rc != 0) fail(FITB_ERR_CUDA, "spectral dt: kernel launch failed");
    if (!(lam > 0.0) || !std::isfinite(lam)) fail(FITB_ERR_STATE, "no live update operator (lambda_max = %g)", lam);
    *lambda_max = lam;
    *dt = safety * 2.0 / std::sqrt(lam);
    if (iterations) *iterations = its;
    H.launches += 5LL * its + 2;
    FITB_CATCH
}

int fitb_set_coeffs_native(fitb_handle* h, const void* alpha_e, const void* beta_e, const void* alpha_h,
                           const void* beta_h, const void* m_eps, const void* m_mu) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!alpha_e || !beta_e || !alpha_h || !beta_h) fail(FITB_ERR_ARG, "null coefficient array");
    auto put = [&](fitb::DevBuf& dst, const void* src, int c0) {
        if (H.prec == 4)
            fitb::pack3<float>(H, (const float*)src, dst.as<float>(), c0);
        else
            fitb::pack3<double>(H, (const double*)src, dst.as<double>(), c0);
    };
    put(H.aE, alpha_e, 0);
    put(H.bE, beta_e, 0);
    put(H.aH, alpha_h, 3);
    put(H.bH, beta_h, 3);
    if (m_eps) put(H.meps, m_eps, 0);
    if (m_mu) put(H.mmu, m_mu, 3);
    const void* arrs[4] = {alpha_e, beta_e, alpha_h, beta_h};
    for (int a = 0; a < 4; ++a) {
        if (H.prec == 4)
            fitb::comp_max(H, (const float*)arrs[a], a < 2 ? 0 : 3, H.coef_max[a]);
        else
            fitb::comp_max(H, (const double*)arrs[a], a < 2 ? 0 : 3, H.coef_max[a]);
    }
    H.coeffs_set = true;
    fitb::compact_coeffs(H);
    H.port_tables_dirty = true;  // the slab step's dead-unit plan reads the coefficients
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_set_coeff_storage(fitb_handle* h, int32_t kind) {
    FITB_TRY
    Handle& H = H_of(h);
    if (kind < fitb::kCoefNative || kind > fitb::kCoefBF16) fail(FITB_ERR_ARG, "coefficient storage kind %d", kind);
    const bool slab = H.stencil_mode == fitb::kModeFused && fitb::is_slab_variant(H.fused_variant);
    if (kind != fitb::kCoefNative && H.stencil_mode != fitb::kModeStream && H.stencil_mode != fitb::kModeVec &&
        !(slab && kind == fitb::kCoefF16 && H.prec == 4))
        fail(FITB_ERR_STATE,
             "compact coefficient storage needs the stream or vec stencil kernels (float16: also the float32 slab "
             "step)");
    H.coef_kind = kind;
    if (kind == fitb::kCoefNative) {
        for (auto& q : H.cq) q.release();
    }
    fitb::plan_stencil(H);
    fitb::compact_coeffs(H);
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_configure_stencil(fitb_handle* h, int32_t kind, int32_t variant, int32_t ichunk) {
    FITB_TRY
    Handle& H = H_of(h);
    if (kind < fitb::kModeSimple || kind > fitb::kModeFused) fail(FITB_ERR_ARG, "stencil kind %d", kind);
    if (ichunk < 0) fail(FITB_ERR_ARG, "ichunk %d", ichunk);
    const bool compact = H.coef_kind != fitb::kCoefNative;
    if (compact && kind != fitb::kModeStream && kind != fitb::kModeVec &&
        !(kind == fitb::kModeFused && fitb::is_slab_variant(variant) && H.coef_kind == fitb::kCoefF16 && H.prec == 4))
        fail(FITB_ERR_STATE,
             "compact coefficient storage needs the stream or vec stencil kernels (float16: also the float32 slab "
             "step)");
    if ((kind == fitb::kModeStream || kind == fitb::kModeVec) && !fitb::stream_batch_supported(H.B))
        fail(FITB_ERR_ARG, "the stream / vec kernels take 1, 2, 4, 8 or 16 field sets, not %d", H.B);
    if (kind == fitb::kModeStream && !fitb::stream_variant_supported(H.B, variant))
        fail(FITB_ERR_ARG, "stream stencil: variant %d / batch %d", variant, H.B);
    if (kind == fitb::kModeVec && (H.B > 8 || variant < 0 || variant > 3))
        fail(FITB_ERR_ARG, "vec stencil: variant %d / batch %d", variant, H.B);
    if (kind == fitb::kModeFused) {
        if (!fitb::fused_variant_ok(H.prec, variant)) fail(FITB_ERR_ARG, "fused variant %d", variant);
        if (H.sibc.present()) fail(FITB_ERR_STATE, "SIBC walls need an in-place stencil mode");
        if (!H.band.empty()) fail(FITB_ERR_STATE, "band DTBC ports need an in-place stencil mode");
        if ((H.disp[0].present() || H.disp[1].present()) && !fitb::is_slab_variant(variant))
            fail(FITB_ERR_STATE,
                 "dispersive materials need an in-place stencil mode or the slab step (fused 16-25)");
        if ((H.disp[0].present() || H.disp[1].present()) && !fitb::disp_clear_of_cpml(H))
            fail(FITB_ERR_STATE, "the slab step takes dispersive materials only outside the CPML slabs");
        if (fitb::is_tile_variant(variant) &&
            !(H.prec == 4 ? fitb::tile_step_fits<float>(fitb::stencil_args<float>(H))
                          : fitb::tile_step_fits<double>(fitb::stencil_args<double>(H))))
            fail(FITB_ERR_ARG, "the tile step does not take this grid / CPML layout");
        if (fitb::is_slab_variant(variant) && H.B % fitb::slab_nb_of(variant - fitb::kFusedSlabBase) != 0)
            fail(FITB_ERR_ARG, "fused variant %d marches %d field sets per CTA: the batch of %d is not a multiple",
                 variant, fitb::slab_nb_of(variant - fitb::kFusedSlabBase), H.B);
        if (fitb::is_slab_variant(variant)) {
            // any march depth the planner may pick: check the deepest and the shallowest
            std::vector<int4> lists[fitb::kSlabLists];
            const int np = H.g.nx + 1;
            std::vector<int> depths;
            for (int c = 12; c <= 20; ++c) depths.push_back(std::min(np, c));
            if (ichunk > 0) depths.push_back(std::min(np, (int)ichunk));
            for (int c : depths)
                if (!fitb::slab_units_of(H, variant, c, lists))
                    fail(FITB_ERR_ARG, "the slab step does not take this grid / CPML layout");
        }
    }
    if (kind == fitb::kModeBulk && H.B != 1) fail(FITB_ERR_ARG, "the bulk-copy stencil takes one field set");
    ck(cudaStreamSynchronize(H.stream), "configure sync");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, H.desc.device);
    if (kind == fitb::kModeBulk) {
        fitb::BulkPlan bp = H.prec == 4 ? fitb::plan_bulk<float>(H.g, sms) : fitb::plan_bulk<double>(H.g, sms);
        if (bp.stages < 3) fail(FITB_ERR_ARG, "the bulk-copy stencil does not fit this grid's rows");
        ck(H.prec == 4 ? fitb::prepare_bulk<float>(bp) : fitb::prepare_bulk<double>(bp), "bulk stencil smem attribute");
        H.plan = bp;
    }
    const size_t blk = (size_t)H.e_block() * H.esz;
    if (kind == fitb::kModeFused) {
        ck(fitb::prepare_fused_any(H.prec, variant), "fused step smem attribute");
        if (!H.e2.p) H.e2.alloc(blk * H.B);
        if (!H.h2.p) H.h2.alloc(blk * H.B);
        for (auto& f : H.faces)
            if (!f->psi2.p) {
                f->psi2.alloc(f->psi.bytes);
                f->dev.psi_next = f->psi2.p;
            }
        H.fused_variant = variant;
    } else if (H.stencil_mode == fitb::kModeFused && H.cur == 1) {
        // leave the fused step with the current fields in the first buffer set
        ck(cudaMemcpyAsync(H.e.p, H.e2.p, blk * H.B, cudaMemcpyDeviceToDevice, H.stream), "fields copy");
        ck(cudaMemcpyAsync(H.h.p, H.h2.p, blk * H.B, cudaMemcpyDeviceToDevice, H.stream), "fields copy");
        for (auto& f : H.faces)
            ck(cudaMemcpyAsync(f->psi.p, f->psi2.p, f->psi.bytes, cudaMemcpyDeviceToDevice, H.stream), "psi copy");
        ck(cudaStreamSynchronize(H.stream), "configure copy sync");
        H.cur = 0;
    }
    if (kind == fitb::kModeVec) H.vec_variant = variant;
    if (kind == fitb::kModeStream) H.stream_variant = compact ? 0 : variant;
    H.stencil_mode = kind;
    fitb::plan_stencil(H);
    if (ichunk > 0) {
        const int nplanes = H.g.nx + 1;
        const int c = std::min(ichunk, nplanes);
        H.ichunk = c;
        H.splan.ichunk = c;
        H.splan.grid_z = (nplanes + c - 1) / c;
    }
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_reserve_steps(fitb_handle* h, int64_t n_steps) {
    FITB_TRY
    Handle& H = H_of(h);
    if (n_steps < 0) fail(FITB_ERR_ARG, "n_steps must be >= 0");
    fitb::ensure_capacity(H, n_steps);
    FITB_CATCH
}

int fitb_device_bytes(fitb_handle* h, int64_t* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!out) fail(FITB_ERR_ARG, "null argument");
    *out = (int64_t)fitb::device_bytes(H);
    FITB_CATCH
}

int fitb_slab_units(fitb_handle* h, int64_t* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!out) fail(FITB_ERR_ARG, "null argument");
    for (int q = 0; q <= fitb::kSlabLists; ++q) out[q] = 0;
    if (H.stencil_mode == fitb::kModeFused && fitb::is_slab_variant(H.fused_variant)) {
        fitb::check_ready(H);
        fitb::refresh_port_tables(H);
        for (int q = 0; q < fitb::kSlabLists; ++q) out[q] = H.n_slab_units[q];
        out[fitb::kSlabLists] = H.n_slab_dead;
    }
    FITB_CATCH
}

int fitb_get_stencil(fitb_handle* h, int32_t* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!out) fail(FITB_ERR_ARG, "null argument");
    const bool planned = H.stencil_mode == fitb::kModeStream || H.stencil_mode == fitb::kModeVec ||
                         H.stencil_mode == fitb::kModeFused;
    out[0] = H.stencil_mode;
    out[1] = H.stencil_mode == fitb::kModeVec     ? H.vec_variant
             : H.stencil_mode == fitb::kModeFused ? H.fused_variant
             : H.stencil_mode == fitb::kModeStream ? H.stream_variant
                                                   : 0;
    out[2] = planned ? H.splan.ichunk : (H.stencil_mode == fitb::kModeBulk ? H.plan.ichunk : H.ichunk);
    out[3] = planned ? H.splan.grid_x : 0;
    out[4] = planned ? H.splan.grid_y : 0;
    out[5] = planned ? H.splan.grid_z : 0;
    FITB_CATCH
}

int fitb_set_fields(fitb_handle* h, int32_t b, const void* e, size_t e_bytes, const void* hf, size_t h_bytes) {
    FITB_TRY
    Handle& H = H_of(h);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    if (e) {
        if (e_bytes != (size_t)H.nE() * H.esz) fail(FITB_ERR_ARG, "e buffer is %zu bytes, expected %zu", e_bytes, (size_t)H.nE() * H.esz);
        if (H.prec == 4)
            fitb::pack3<float>(H, (const float*)e, H.Ec().as<float>() + (long long)b * H.e_block(), 0);
        else
            fitb::pack3<double>(H, (const double*)e, H.Ec().as<double>() + (long long)b * H.e_block(), 0);
    }
    if (hf) {
        if (h_bytes != (size_t)H.nH() * H.esz) fail(FITB_ERR_ARG, "h buffer is %zu bytes, expected %zu", h_bytes, (size_t)H.nH() * H.esz);
        if (H.prec == 4)
            fitb::pack3<float>(H, (const float*)hf, H.Hc().as<float>() + (long long)b * H.e_block(), 3);
        else
            fitb::pack3<double>(H, (const double*)hf, H.Hc().as<double>() + (long long)b * H.e_block(), 3);
    }
    H.skip_sync = H.n_slab_dead > 0;
    FITB_CATCH
}

int fitb_read_fields(fitb_handle* h, int32_t b, void* e, size_t e_bytes, void* hf, size_t h_bytes) {
    FITB_TRY
    Handle& H = H_of(h);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    if (e) {
        if (e_bytes != (size_t)H.nE() * H.esz) fail(FITB_ERR_ARG, "e buffer size mismatch");
        if (H.prec == 4)
            fitb::unpack3<float>(H, H.Ec().as<float>() + (long long)b * H.e_block(), (float*)e, 0);
        else
            fitb::unpack3<double>(H, H.Ec().as<double>() + (long long)b * H.e_block(), (double*)e, 0);
    }
    if (hf) {
        if (h_bytes != (size_t)H.nH() * H.esz) fail(FITB_ERR_ARG, "h buffer size mismatch");
        if (H.prec == 4)
            fitb::unpack3<float>(H, H.Hc().as<float>() + (long long)b * H.e_block(), (float*)hf, 3);
        else
            fitb::unpack3<double>(H, H.Hc().as<double>() + (long long)b * H.e_block(), (double*)hf, 3);
    }
    FITB_CATCH
}

int fitb_add_cpml(fitb_handle* h, int32_t face, int32_t n_pml, const double* b, const double* c, const double* ck_,
                  const uint8_t* air_e1, const uint8_t* air_e2, const uint8_t* air_h1, const uint8_t* air_h2) {
    FITB_TRY
    Handle& H = H_of(h);
    if (face < 0 || face > 5) fail(FITB_ERR_ARG, "face must be 0..5");
    if (!b || !c || !ck_) fail(FITB_ERR_ARG, "null CPML table");
    if ((int)H.faces.size() >= fitb::kMaxFaces) fail(FITB_ERR_LIMIT, "at most %d CPML faces", fitb::kMaxFaces);
    for (auto& f : H.faces)
        if (f->face == face) fail(FITB_ERR_ARG, "CPML face %d already added", face);
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "boundaries must be added before the first step");
    const uint8_t* air[4] = {air_e1, air_e2, air_h1, air_h2};
    if (H.prec == 4)
        fitb::add_cpml_impl<float>(H, face, n_pml, b, c, ck_, air);
    else
        fitb::add_cpml_impl<double>(H, face, n_pml, b, c, ck_, air);
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_add_lumped(fitb_handle* h, int32_t n_edges, const int64_t* flat_e_idx, const double* signs,
                    const double* betas, double r, double l, double c, double record_scale, int32_t* out_id) {
    FITB_TRY
    Handle& H = H_of(h);
    if (n_edges < 1 || !flat_e_idx || !signs || !betas) fail(FITB_ERR_ARG, "lumped port needs >= 1 edge");
    if (r < 0 && l < 0 && c < 0) fail(FITB_ERR_ARG, "lumped element needs at least one of R, L, C");
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "ports must be added before the first step");
    auto lp = std::make_unique<fitb::LumpedHost>();
    std::vector<long long> off((size_t)n_edges);
    double bsum = 0.0;
    for (int q = 0; q < n_edges; ++q) {
        off[(size_t)q] = H.flat_to_off(false, flat_e_idx[q]);
        bsum += betas[q];
    }
    fitb::upload(lp->off, off);
    lp->off_host = off;
    fitb::upload(lp->sign, std::vector<double>(signs, signs + n_edges));
    fitb::upload(lp->beta, std::vector<double>(betas, betas + n_edges));
    lp->st.alloc(sizeof(double) * 4 * H.B);
    lp->src_host.assign((size_t)H.B, 0.0);
    fitb::upload(lp->src, lp->src_host);
    fitb::LumpedDev& d = lp->dev;
    d.n_edges = n_edges;
    d.off = lp->off.as<long long>();
    d.sign = lp->sign.as<double>();
    d.beta = lp->beta.as<double>();
    d.beta_sum = bsum;
    d.R = r;
    d.L = l;
    d.C = c;
    d.rec_scale = record_scale;
    d.src = lp->src.as<double>();
    d.n_src = 1;
    d.st = lp->st.as<double>();
    d.channel = H.nch;
    H.nch += 1;
    if (out_id) *out_id = (int32_t)H.lumped.size();
    H.lumped.push_back(std::move(lp));
    H.cap = 0;
    H.recV.release();
    H.recI.release();
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_set_lumped_source(fitb_handle* h, int32_t id, int32_t b, int64_t n_samples, const double* v_src) {
    FITB_TRY
    Handle& H = H_of(h);
    if (id < 0 || id >= (int)H.lumped.size()) fail(FITB_ERR_ARG, "lumped port %d does not exist", id);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    if (n_samples < 0 || (n_samples > 0 && !v_src)) fail(FITB_ERR_ARG, "bad source samples");
    fitb::LumpedHost& lp = *H.lumped[id];
    long long n_old = lp.dev.n_src;
    long long n_new = std::max<long long>(n_old, std::max<int64_t>(n_samples, 1));
    std::vector<double> tab((size_t)(H.B * n_new), 0.0);
    for (int q = 0; q < H.B; ++q)
        for (long long t = 0; t < n_old; ++t) tab[(size_t)(q * n_new + t)] = lp.src_host[(size_t)(q * n_old + t)];
    for (long long t = 0; t < n_new; ++t) tab[(size_t)(b * n_new + t)] = t < n_samples ? v_src[t] : 0.0;
    lp.src_host = tab;
    fitb::upload(lp.src, tab);
    lp.dev.src = lp.src.as<double>();
    lp.dev.n_src = n_new;
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_push_lumped_samples(fitb_handle* h, int32_t id, int32_t b, int64_t step0, int64_t n, const double* host) {
    FITB_TRY
    Handle& H = H_of(h);
    if (id < 0 || id >= (int)H.lumped.size()) fail(FITB_ERR_ARG, "lumped port %d does not exist", id);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    fitb::LumpedHost& lp = *H.lumped[id];
    if (n < 0 || step0 < 0 || step0 + n > lp.dev.n_src || (n > 0 && !host))
        fail(FITB_ERR_ARG, "samples [%lld, %lld) outside the source table of %lld", (long long)step0,
             (long long)(step0 + n), lp.dev.n_src);
    if (n == 0) return FITB_OK;
    ck(cudaMemcpyAsync(lp.src.as<double>() + (size_t)b * lp.dev.n_src + step0, host, (size_t)n * sizeof(double),
                       cudaMemcpyHostToDevice, H.stream),
       "push samples");
    FITB_CATCH
}

int fitb_add_modal_port(fitb_handle* h, const fitb_modal_desc* d, int32_t* out_id) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!d) fail(FITB_ERR_ARG, "null descriptor");
    if (d->n_modes < 1 || d->n_modes > fitb::kMaxModes) fail(FITB_ERR_LIMIT, "n_modes must be 1..%d", fitb::kMaxModes);
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "ports must be added before the first step");
    const int M = d->n_modes;
    const int ne = d->n_e_u + d->n_e_v, nh = d->n_h_u + d->n_h_v;
    if (ne < 1) fail(FITB_ERR_ARG, "modal port without plane samples");
    if (!d->port_e_idx || !d->int_e_idx || !d->me_port || !d->me_int || !d->e_profile || !d->v_profile ||
        !d->mur_r || !d->tau || !d->record_scale || !d->is_dtbc)
        fail(FITB_ERR_ARG, "modal descriptor has a null array");
    if (nh > 0 && (!d->port_h_idx || !d->mh_port || !d->h_profile)) fail(FITB_ERR_ARG, "modal descriptor: null H arrays");
    auto mp = std::make_unique<fitb::ModalHost>();
    mp->n_modes = M;
    std::vector<long long> pe((size_t)ne), ie((size_t)ne), ph((size_t)nh);
    for (int p = 0; p < ne; ++p) {
        pe[(size_t)p] = H.flat_to_off(false, d->port_e_idx[p]);
        ie[(size_t)p] = H.flat_to_off(false, d->int_e_idx[p]);
    }
    for (int p = 0; p < nh; ++p) ph[(size_t)p] = H.flat_to_off(true, d->port_h_idx[p]);
    fitb::upload(mp->port_e, pe);
    mp->port_e_host = pe;
    fitb::upload(mp->int_e, ie);
    fitb::upload(mp->port_h, ph);
    fitb::upload(mp->me_port, std::vector<double>(d->me_port, d->me_port + ne));
    fitb::upload(mp->me_int, std::vector<double>(d->me_int, d->me_int + ne));
    fitb::upload(mp->mh_port, nh ? std::vector<double>(d->mh_port, d->mh_port + nh) : std::vector<double>(1, 0.0));
    fitb::upload(mp->eprof, std::vector<double>(d->e_profile, d->e_profile + (size_t)M * ne));
    fitb::upload(mp->vprof, std::vector<double>(d->v_profile, d->v_profile + (size_t)M * ne));
    fitb::upload(mp->hprof, nh ? std::vector<double>(d->h_profile, d->h_profile + (size_t)M * nh) : std::vector<double>(1, 0.0));
    bool any_mur = false;
    fitb::ModalDev& md = mp->dev;
    md.n_modes = M;
    md.n_e = ne;
    md.n_e_u = d->n_e_u;
    md.n_h = nh;
    md.n_h_u = d->n_h_u;
    md.dt = H.dt;
    mp->n_tables_mode.assign((size_t)M, 0);
    mp->ktabs.assign((size_t)M, {});
    mp->dtbc_r.assign((size_t)M, 0.0);
    mp->dtbc_q.assign((size_t)M, 0.0);
    for (int m = 0; m < M; ++m) {
        md.mur_r[m] = d->mur_r[m];
        md.tau[m] = d->tau[m];
        md.rec_scale[m] = d->record_scale[m];
        md.is_dtbc[m] = d->is_dtbc[m] ? 1 : 0;
        if (md.is_dtbc[m]) {
            if (!d->dtbc_r || !d->dtbc_q) fail(FITB_ERR_ARG, "DTBC mode without r/q");
            md.r2[m] = d->dtbc_r[m] * d->dtbc_r[m];
            md.q2[m] = d->dtbc_q[m] * d->dtbc_q[m];
            mp->dtbc_r[(size_t)m] = d->dtbc_r[m];
            mp->dtbc_q[(size_t)m] = d->dtbc_q[m];
        } else {
            any_mur = true;
        }
    }
    int n0 = d->dtbc_n_kernel_init > 0 ? d->dtbc_n_kernel_init : 4096;
    md.n0 = n0;
    md.comp_on = (d->has_complement && any_mur) ? 1 : 0;
    if (d->has_complement) {
        if (!d->comp_r || !d->comp_live) fail(FITB_ERR_ARG, "complement absorber arrays missing");
        fitb::upload(mp->comp_r, std::vector<double>(d->comp_r, d->comp_r + ne));
        fitb::upload(mp->comp_live, std::vector<double>(d->comp_live, d->comp_live + ne));
    }
    mp->st.alloc(sizeof(double) * H.B * 4 * fitb::kMaxModes);
    mp->comp_state.alloc(sizeof(double) * H.B * 2 * ne);
    mp->scratch.alloc(sizeof(double) * H.B * 2 * ne);
    // a plane larger than one chunk runs its projections and reconstruction
    // over many CTAs (FITB_PORT_CHUNK overrides the chunk size, 32 .. 2^20)
    {
        int chunk = fitb::kPortChunk;
        if (const char* t = std::getenv("FITB_PORT_CHUNK")) chunk = std::max(32, std::min(1 << 20, atoi(t)));
        const long long nmax = std::max<long long>(ne, nh);
        md.chunk = chunk;
        md.n_chunks = ne > chunk ? (int)((nmax + chunk - 1) / chunk) : 1;
        if (md.n_chunks > 1) {
            std::vector<double> zero((size_t)H.B * md.n_chunks * 3 * fitb::kMaxModes, 0.0);
            fitb::upload(mp->part, zero);
            fitb::upload(mp->vals, std::vector<double>((size_t)H.B * 2 * fitb::kMaxModes, 0.0));
            fitb::upload(mp->done, std::vector<int>((size_t)H.B, 0));
            md.part = mp->part.as<double>();
            md.vals = mp->vals.as<double>();
            md.done = mp->done.as<int>();
        }
        H.modal_chunks = std::max(H.modal_chunks, md.n_chunks);
    }
    mp->exc_host.assign((size_t)H.B, -1);
    mp->buflen_host.assign((size_t)H.B, 5);
    mp->n_wf = 1;
    mp->wf_host.assign((size_t)H.B, 0.0);
    fitb::upload(mp->exc, mp->exc_host);
    fitb::upload(mp->buflen, mp->buflen_host);
    fitb::upload(mp->wf, mp->wf_host);
    md.port_e = mp->port_e.as<long long>();
    md.int_e = mp->int_e.as<long long>();
    md.port_h = mp->port_h.as<long long>();
    md.me_port = mp->me_port.as<double>();
    md.me_int = mp->me_int.as<double>();
    md.mh_port = mp->mh_port.as<double>();
    md.eprof = mp->eprof.as<double>();
    md.vprof = mp->vprof.as<double>();
    md.hprof = mp->hprof.as<double>();
    md.comp_r = mp->comp_r.as<double>();
    md.comp_live = mp->comp_live.as<double>();
    md.st = mp->st.as<double>();
    md.comp_state = mp->comp_state.as<double>();
    md.scratch = mp->scratch.as<double>();
    md.exc_mode = mp->exc.as<int>();
    md.wf = mp->wf.as<double>();
    md.n_wf = 1;
    md.buf_len = mp->buflen.as<int>();
    md.channel0 = H.nch;
    H.nch += M;
    if (out_id) *out_id = (int32_t)H.modal.size();
    // history buffers are (re)allocated by ensure_capacity
    long long want = std::max<long long>(H.cap, d->max_steps > 0 ? d->max_steps : 1024);
    H.modal.push_back(std::move(mp));
    H.cap = 0;
    H.recV.release();
    H.recI.release();
    for (auto& other : H.modal) {
        other->whist.release();
        other->shist.release();
    }
    fitb::ensure_capacity(H, want);
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_set_dtbc_kernel(fitb_handle* h, int32_t port, int32_t mode, int32_t n_kernel, const double* l) {
    FITB_TRY
    Handle& H = H_of(h);
    if (port < 0 || port >= (int)H.modal.size()) fail(FITB_ERR_ARG, "modal port %d does not exist", port);
    fitb::ModalHost& mp = *H.modal[port];
    if (mode < 0 || mode >= mp.n_modes || !mp.dev.is_dtbc[mode]) fail(FITB_ERR_ARG, "mode %d is not a DTBC mode", mode);
    if (!l) fail(FITB_ERR_ARG, "null kernel");
    // Tables are appended in order n0, 2 n0, 4 n0, ...
    long long expect = (long long)mp.dev.n0 << mp.n_tables_mode[(size_t)mode];
    if (n_kernel != expect) fail(FITB_ERR_ARG, "expected the DTBC table of length %lld next, got %d", expect, n_kernel);
    auto& tab = mp.ktabs[(size_t)mode];
    tab.insert(tab.end(), l, l + n_kernel);
    mp.n_tables_mode[(size_t)mode] += 1;
    fitb::upload(mp.ktab[mode], tab);
    mp.dev.ktab[mode] = mp.ktab[mode].as<double>();
    mp.dev.n_tables = *std::max_element(mp.n_tables_mode.begin(), mp.n_tables_mode.end());
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_build_dtbc_kernel(fitb_handle* h, int32_t port, int32_t mode, int64_t n_steps) {
    FITB_TRY
    Handle& H = H_of(h);
    if (port < 0 || port >= (int)H.modal.size()) fail(FITB_ERR_ARG, "modal port %d does not exist", port);
    fitb::ModalHost& mp = *H.modal[port];
    if (mode < 0 || mode >= mp.n_modes || !mp.dev.is_dtbc[mode]) fail(FITB_ERR_ARG, "mode %d is not a DTBC mode", mode);
    if (n_steps < 1) fail(FITB_ERR_ARG, "n_steps must be >= 1");
    if (mp.dev.n0 < 2) fail(FITB_ERR_STATE, "the port's initial DTBC kernel length is unset");
    // the tables a run of n_steps chain steps visits: n0, 2 n0, ... up to the
    // first length >= n_steps (dtbc.py:351-363), those not yet set
    std::vector<long long> lens;
    for (long long L = mp.dev.n0;; L *= 2) {
        lens.push_back(L);
        if (L >= n_steps) break;
    }
    const size_t have = (size_t)mp.n_tables_mode[(size_t)mode];
    if (have >= lens.size()) return FITB_OK;
    if (lens.back() > (1LL << 26)) fail(FITB_ERR_LIMIT, "DTBC kernel of %lld entries", lens.back());
    fitb::DevBuf x, l;
    x.alloc((size_t)(8 * lens.back()) * sizeof(double2), false);
    l.alloc((size_t)lens.back() * sizeof(double), false);
    std::vector<double> host;
    for (size_t t = have; t < lens.size(); ++t) {
        const int n = (int)lens[t];
        fitb::launch_dtbc_kernel(mp.dtbc_r[(size_t)mode], mp.dtbc_q[(size_t)mode], n, x.as<double2>(), l.as<double>(),
                                 H.stream);
        H.launches += 2;
        ck(cudaGetLastError(), "DTBC kernel launch");
        host.resize((size_t)n);
        ck(cudaMemcpyAsync(host.data(), l.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, H.stream),
           "DTBC kernel D2H");
        ck(cudaStreamSynchronize(H.stream), "DTBC kernel sync");
        auto& tab = mp.ktabs[(size_t)mode];
        tab.insert(tab.end(), host.begin(), host.end());
        mp.n_tables_mode[(size_t)mode] += 1;
    }
    fitb::upload(mp.ktab[mode], mp.ktabs[(size_t)mode]);
    mp.dev.ktab[mode] = mp.ktab[mode].as<double>();
    mp.dev.n_tables = *std::max_element(mp.n_tables_mode.begin(), mp.n_tables_mode.end());
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_set_modal_source(fitb_handle* h, int32_t port, int32_t b, int32_t mode, int64_t n_samples, const double* w) {
    FITB_TRY
    Handle& H = H_of(h);
    if (port < 0 || port >= (int)H.modal.size()) fail(FITB_ERR_ARG, "modal port %d does not exist", port);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    fitb::ModalHost& mp = *H.modal[port];
    if (mode < -1 || mode >= mp.n_modes) fail(FITB_ERR_ARG, "mode_idx %d out of range [0, %d)", mode, mp.n_modes);
    if (mode >= 0 && (n_samples < 1 || !w)) fail(FITB_ERR_ARG, "excitation needs waveform samples");
    mp.exc_host[(size_t)b] = mode;
    if (mode >= 0) {
        // set_excitation: buf_len = max(ceil((tau + dt) / dt) + 3, 5)
        double tau = mp.dev.tau[mode];
        int bl = (int)std::ceil((tau + H.dt) / H.dt) + 3;
        mp.buflen_host[(size_t)b] = std::max(bl, 5);
        long long n_old = mp.n_wf, n_new = std::max<long long>(n_old, n_samples);
        std::vector<double> tab((size_t)(H.B * n_new), 0.0);
        for (int q = 0; q < H.B; ++q)
            for (long long t = 0; t < n_old; ++t) tab[(size_t)(q * n_new + t)] = mp.wf_host[(size_t)(q * n_old + t)];
        for (long long t = 0; t < n_new; ++t) tab[(size_t)(b * n_new + t)] = t < n_samples ? w[t] : 0.0;
        mp.wf_host = tab;
        mp.n_wf = n_new;
        fitb::upload(mp.wf, tab);
        mp.dev.wf = mp.wf.as<double>();
        mp.dev.n_wf = n_new;
    }
    fitb::upload(mp.exc, mp.exc_host);
    fitb::upload(mp.buflen, mp.buflen_host);
    mp.dev.exc_mode = mp.exc.as<int>();
    mp.dev.buf_len = mp.buflen.as<int>();
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_add_dispersion_block(fitb_handle* h, int32_t side, int64_t n_states, const int64_t* idx, const double* g,
                              int32_t n_poles, const int32_t* kind, const double* k_re, const double* k_im,
                              const double* c_re, const double* c_im, const double* weight) {
    FITB_TRY
    Handle& H = H_of(h);
    if (side != 0 && side != 1) fail(FITB_ERR_ARG, "dispersion side %d (0 = E, 1 = H)", side);
    if (n_states < 1 || n_poles < 1 || !idx || !g || !kind || !k_re || !k_im || !c_re || !c_im || !weight)
        fail(FITB_ERR_ARG, "dispersion block needs states, poles and all arrays");
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "dispersion must be added before the first step");
    if (H.stencil_mode == fitb::kModeFused && !fitb::is_slab_variant(H.fused_variant))
        fail(FITB_ERR_STATE, "dispersive materials need an in-place stencil mode or the slab step (fused 16-25)");
    fitb::DispHost& D = H.disp[side];
    const int blk = (int)D.pole_start.size() - 1;
    for (int q = 0; q < n_poles; ++q) {
        if (kind[q] != 0 && kind[q] != 1) fail(FITB_ERR_ARG, "pole kind %d", kind[q]);
        D.kind.push_back(kind[q]);
        D.k_re.push_back(k_re[q]);
        D.k_im.push_back(k_im[q]);
        D.c_re.push_back(c_re[q]);
        D.c_im.push_back(c_im[q]);
        D.opk_re.push_back(1.0 + k_re[q]);
        D.opk_im.push_back(kind[q] ? k_im[q] : 0.0);
        D.hw.push_back(0.5 * weight[q]);
    }
    D.pole_start.push_back(D.pole_start.back() + n_poles);
    for (int64_t s = 0; s < n_states; ++s) {
        D.off.push_back(H.flat_to_off(side == 1, idx[s]));
        D.g.push_back(g[s]);
        D.state_block.push_back(blk);
        D.slot.push_back(D.n_slots);
        D.n_slots += 2LL * n_poles;
    }
    // entries shared by several blocks take their terms in block order
    const long long ns = (long long)D.off.size();
    std::vector<long long> order((size_t)ns);
    for (long long s = 0; s < ns; ++s) order[(size_t)s] = s;
    std::stable_sort(order.begin(), order.end(), [&](long long a, long long b) { return D.off[(size_t)a] < D.off[(size_t)b]; });
    std::vector<long long> uoff, ustate;
    std::vector<int> ustart;
    for (size_t r = 0; r < order.size(); ++r) {
        const long long st = order[r];
        if (r == 0 || D.off[(size_t)st] != uoff.back()) {
            uoff.push_back(D.off[(size_t)st]);
            ustart.push_back((int)ustate.size());
        }
        ustate.push_back(st);
    }
    ustart.push_back((int)ustate.size());
    // device tables
    fitb::upload(D.d_off, D.off);
    if (H.prec == 4)
        fitb::upload(D.d_g, fitb::cast_vec<float>(D.g.data(), ns));
    else
        fitb::upload(D.d_g, D.g);
    fitb::upload(D.d_state_block, D.state_block);
    fitb::upload(D.d_slot, D.slot);
    fitb::upload(D.d_pole_start, D.pole_start);
    fitb::upload(D.d_kind, D.kind);
    for (auto pr : {std::make_pair(&D.d_k_re, &D.k_re), std::make_pair(&D.d_k_im, &D.k_im),
                    std::make_pair(&D.d_c_re, &D.c_re), std::make_pair(&D.d_c_im, &D.c_im),
                    std::make_pair(&D.d_opk_re, &D.opk_re), std::make_pair(&D.d_opk_im, &D.opk_im),
                    std::make_pair(&D.d_hw, &D.hw)})
        fitb::upload(*pr.first, *pr.second);
    fitb::upload(D.d_uoff, uoff);
    fitb::upload(D.d_ustart, ustart);
    fitb::upload(D.d_ustate, ustate);
    D.d_J.alloc((size_t)H.B * D.n_slots * H.esz);
    D.d_fprev.alloc((size_t)H.B * ns * H.esz);
    fitb::DispDev& dv = D.dev;
    dv.n_states = ns;
    dv.off = D.d_off.as<long long>();
    dv.g = D.d_g.p;
    dv.state_block = D.d_state_block.as<int>();
    dv.slot = D.d_slot.as<long long>();
    dv.n_slots = D.n_slots;
    dv.J = D.d_J.p;
    dv.fprev = D.d_fprev.p;
    dv.pole_start = D.d_pole_start.as<int>();
    dv.kind = D.d_kind.as<int>();
    dv.k_re = D.d_k_re.as<double>();
    dv.k_im = D.d_k_im.as<double>();
    dv.c_re = D.d_c_re.as<double>();
    dv.c_im = D.d_c_im.as<double>();
    dv.opk_re = D.d_opk_re.as<double>();
    dv.opk_im = D.d_opk_im.as<double>();
    dv.hw = D.d_hw.as<double>();
    dv.n_unique = (long long)uoff.size();
    dv.uoff = D.d_uoff.as<long long>();
    dv.ustart = D.d_ustart.as<int>();
    dv.ustate = D.d_ustate.as<long long>();
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_add_band_port(fitb_handle* h, const fitb_band_desc* d, int32_t* out_id) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!d || !out_id) fail(FITB_ERR_ARG, "null argument");
    const int p = d->p, M = d->n_modes;
    if (p < 1 || p > fitb::kBandPMax) fail(FITB_ERR_LIMIT, "band port rank p = %d (1..%d)", p, fitb::kBandPMax);
    if (M < 1 || M > fitb::kMaxModes) fail(FITB_ERR_LIMIT, "band port channels %d (1..%d)", M, fitb::kMaxModes);
    if (d->n_kernel_init < 2) fail(FITB_ERR_ARG, "n_kernel_init must be >= 2");
    if (d->n_u < 0 || d->n_v < 0 || d->n_u + d->n_v < 1 || d->n1 < 1 || d->n_h < 0)
        fail(FITB_ERR_ARG, "band port sizes");
    if (!d->e_u_idx && d->n_u > 0) fail(FITB_ERR_ARG, "null e_u_idx");
    if (!d->e_v_idx && d->n_v > 0) fail(FITB_ERR_ARG, "null e_v_idx");
    if (!d->x1_idx || !d->M_coup || !d->D0 || !d->Dm1 || !d->me || !d->v_profile || !d->record_scale ||
        (d->n_u > 0 && !d->Wu) || (d->n_v > 0 && !d->Wv) || (d->n_h > 0 && (!d->h_idx || !d->mh || !d->h_profile)))
        fail(FITB_ERR_ARG, "band port arrays");
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "ports must be added before the first step");
    if (H.stencil_mode == fitb::kModeFused) fail(FITB_ERR_STATE, "band DTBC ports need an in-place stencil mode");
    const long long ne = H.nE(), nh = H.nH();
    auto offs = [&](const int64_t* idx, long long n, bool is_h) {
        std::vector<long long> o((size_t)std::max<long long>(n, 1), 0);
        for (long long q = 0; q < n; ++q) {
            if (idx[q] < 0 || idx[q] >= (is_h ? nh : ne)) fail(FITB_ERR_ARG, "band port index %lld out of range", (long long)idx[q]);
            o[(size_t)q] = H.flat_to_off(is_h, idx[q]);
        }
        return o;
    };
    auto vec = [](const double* a, long long n) {
        return n > 0 ? std::vector<double>(a, a + n) : std::vector<double>(1, 0.0);
    };
    auto bp = std::make_unique<fitb::BandHost>();
    bp->p = p;
    const long long nt = d->n_u + d->n_v;
    fitb::upload(bp->eu, offs(d->e_u_idx, d->n_u, false));
    fitb::upload(bp->ev, offs(d->e_v_idx, d->n_v, false));
    fitb::upload(bp->x1, offs(d->x1_idx, d->n1, false));
    fitb::upload(bp->hh, offs(d->h_idx, d->n_h, true));
    fitb::upload(bp->Wu, vec(d->Wu, d->n_u * p));
    fitb::upload(bp->Wv, vec(d->Wv, d->n_v * p));
    fitb::upload(bp->Mc, vec(d->M_coup, (long long)p * d->n1));
    fitb::upload(bp->D0, vec(d->D0, (long long)p * p));
    fitb::upload(bp->Dm1, vec(d->Dm1, (long long)p * p));
    fitb::upload(bp->me, vec(d->me, nt));
    fitb::upload(bp->vprof, vec(d->v_profile, (long long)M * nt));
    fitb::upload(bp->mh, vec(d->mh, d->n_h));
    fitb::upload(bp->hprof, vec(d->h_profile, (long long)M * d->n_h));
    fitb::upload(bp->rec_scale, vec(d->record_scale, M));
    bp->st.alloc((size_t)H.B * 2 * p * sizeof(double));
    std::vector<double> x1p((size_t)H.B * d->n1, 0.0);
    if (d->x1_prev0)
        for (int b = 0; b < H.B; ++b)
            for (long long q = 0; q < d->n1; ++q) x1p[(size_t)(b * d->n1 + q)] = d->x1_prev0[q];
    fitb::upload(bp->x1prev, x1p);
    bp->src_on_host.assign((size_t)H.B, 0);
    fitb::upload(bp->src_on, bp->src_on_host);
    fitb::upload(bp->src, std::vector<double>(1, 0.0));
    fitb::upload(bp->kout, std::vector<double>(1, 0.0));
    fitb::upload(bp->kin, std::vector<double>(1, 0.0));
    fitb::BandDev& dv = bp->dev;
    dv.p = p;
    dv.M = M;
    dv.channel0 = H.nch;
    dv.n_u = d->n_u;
    dv.n_v = d->n_v;
    dv.n1 = d->n1;
    dv.n_h = d->n_h;
    dv.eu = bp->eu.as<long long>();
    dv.ev = bp->ev.as<long long>();
    dv.x1 = bp->x1.as<long long>();
    dv.hh = bp->hh.as<long long>();
    dv.Wu = bp->Wu.as<double>();
    dv.Wv = bp->Wv.as<double>();
    dv.Mc = bp->Mc.as<double>();
    dv.D0 = bp->D0.as<double>();
    dv.Dm1 = bp->Dm1.as<double>();
    dv.me = bp->me.as<double>();
    dv.vprof = bp->vprof.as<double>();
    dv.mh = bp->mh.as<double>();
    dv.hprof = bp->hprof.as<double>();
    dv.rec_scale = bp->rec_scale.as<double>();
    dv.n0 = d->n_kernel_init;
    dv.st = bp->st.as<double>();
    dv.x1prev = bp->x1prev.as<double>();
    H.nch += M;
    *out_id = (int32_t)H.band.size();
    H.band.push_back(std::move(bp));
    // the recorder and the histories are sized for the new channel count
    H.cap = 0;
    fitb::ensure_capacity(H, 1);
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_set_band_kernel(fitb_handle* h, int32_t port, int32_t incoming, int32_t n_kernel, const double* L) {
    FITB_TRY
    Handle& H = H_of(h);
    if (port < 0 || port >= (int)H.band.size()) fail(FITB_ERR_ARG, "band port %d does not exist", port);
    if (!L) fail(FITB_ERR_ARG, "null kernel");
    fitb::BandHost& bp = *H.band[port];
    int& nt = incoming ? bp.n_in : bp.n_out;
    const long long expect = bp.dev.n0 << nt;
    if (n_kernel != expect) fail(FITB_ERR_ARG, "expected the band kernel table of length %lld next, got %d", expect, n_kernel);
    auto& tab = incoming ? bp.kin_host : bp.kout_host;
    tab.insert(tab.end(), L, L + (size_t)n_kernel * bp.p * bp.p);
    nt += 1;
    fitb::upload(incoming ? bp.kin : bp.kout, tab);
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_set_band_source(fitb_handle* h, int32_t port, int32_t b, int64_t n_samples, const double* src) {
    FITB_TRY
    Handle& H = H_of(h);
    if (port < 0 || port >= (int)H.band.size()) fail(FITB_ERR_ARG, "band port %d does not exist", port);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    if (n_samples < 1 || !src) fail(FITB_ERR_ARG, "band source needs samples");
    fitb::BandHost& bp = *H.band[port];
    const int p = bp.p;
    const long long n_old = bp.n_src, n_new = std::max<long long>(n_old, n_samples);
    std::vector<double> tab((size_t)(H.B * n_new * p), 0.0);
    for (int q = 0; q < H.B; ++q)
        for (long long t = 0; t < n_old; ++t)
            for (int i = 0; i < p; ++i)
                tab[(size_t)((q * n_new + t) * p + i)] = bp.src_host[(size_t)((q * n_old + t) * p + i)];
    for (long long t = 0; t < n_new; ++t)
        for (int i = 0; i < p; ++i) tab[(size_t)((b * n_new + t) * p + i)] = t < n_samples ? src[t * p + i] : 0.0;
    bp.src_host = tab;
    bp.n_src = n_new;
    bp.src_on_host[(size_t)b] = 1;
    fitb::upload(bp.src, tab);
    fitb::upload(bp.src_on, bp.src_on_host);
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_add_sibc_block(fitb_handle* h, int64_t n_faces, const int64_t* idx, const double* g, int32_t n_branches,
                        const double* k, const double* q) {
    FITB_TRY
    Handle& H = H_of(h);
    if (n_faces < 1 || !idx || !g || n_branches < 0 || (n_branches > 0 && (!k || !q)))
        fail(FITB_ERR_ARG, "SIBC block needs faces, their g and the branch constants");
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "SIBC walls must be added before the first step");
    if (H.stencil_mode == fitb::kModeFused) fail(FITB_ERR_STATE, "SIBC walls need an in-place stencil mode");
    const long long nh = H.nH();
    for (int64_t s = 0; s < n_faces; ++s)
        if (idx[s] < 0 || idx[s] >= nh) fail(FITB_ERR_ARG, "SIBC face index %lld out of range", (long long)idx[s]);
    fitb::SibcHost& S = H.sibc;
    const int blk = (int)S.br_start.size() - 1;
    for (int p = 0; p < n_branches; ++p) {
        S.k.push_back(k[p]);
        S.q.push_back(q[p]);
        S.hopk.push_back(0.5 * (1.0 + k[p]));
    }
    S.br_start.push_back(S.br_start.back() + n_branches);
    for (int64_t f = 0; f < n_faces; ++f) {
        S.off.push_back(H.flat_to_off(true, idx[f]));
        S.g.push_back(g[f]);
        S.state_block.push_back(blk);
        S.slot.push_back(S.n_slots);
        S.n_slots += n_branches;
    }
    // faces booked by several walls take their terms in wall order
    const long long ns = (long long)S.off.size();
    std::vector<long long> order((size_t)ns);
    for (long long t = 0; t < ns; ++t) order[(size_t)t] = t;
    std::stable_sort(order.begin(), order.end(), [&](long long a, long long b) { return S.off[(size_t)a] < S.off[(size_t)b]; });
    std::vector<long long> uoff, ustate;
    std::vector<int> ustart;
    for (size_t r = 0; r < order.size(); ++r) {
        const long long st = order[r];
        if (r == 0 || S.off[(size_t)st] != uoff.back()) {
            uoff.push_back(S.off[(size_t)st]);
            ustart.push_back((int)ustate.size());
        }
        ustate.push_back(st);
    }
    ustart.push_back((int)ustate.size());
    fitb::upload(S.d_off, S.off);
    if (H.prec == 4)
        fitb::upload(S.d_g, fitb::cast_vec<float>(S.g.data(), ns));
    else
        fitb::upload(S.d_g, S.g);
    fitb::upload(S.d_state_block, S.state_block);
    fitb::upload(S.d_slot, S.slot);
    fitb::upload(S.d_br_start, S.br_start);
    // zero-length tables still get a valid pointer
    fitb::upload(S.d_k, S.k.empty() ? std::vector<double>(1, 0.0) : S.k);
    fitb::upload(S.d_q, S.q.empty() ? std::vector<double>(1, 0.0) : S.q);
    fitb::upload(S.d_hopk, S.hopk.empty() ? std::vector<double>(1, 0.0) : S.hopk);
    fitb::upload(S.d_uoff, uoff);
    fitb::upload(S.d_ustart, ustart);
    fitb::upload(S.d_ustate, ustate);
    S.d_u.alloc((size_t)H.B * std::max<long long>(S.n_slots, 1) * H.esz);
    S.d_hprev.alloc((size_t)H.B * ns * H.esz);
    fitb::SibcDev& dv = S.dev;
    dv.n_states = ns;
    dv.off = S.d_off.as<long long>();
    dv.g = S.d_g.p;
    dv.state_block = S.d_state_block.as<int>();
    dv.slot = S.d_slot.as<long long>();
    dv.n_slots = S.n_slots;
    dv.u = S.d_u.p;
    dv.hprev = S.d_hprev.p;
    dv.br_start = S.d_br_start.as<int>();
    dv.k = S.d_k.as<double>();
    dv.q = S.d_q.as<double>();
    dv.hopk = S.d_hopk.as<double>();
    dv.n_unique = (long long)uoff.size();
    dv.uoff = S.d_uoff.as<long long>();
    dv.ustart = S.d_ustart.as<int>();
    dv.ustate = S.d_ustate.as<long long>();
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_add_plane_wave(fitb_handle* h, const fitb_plane_wave_desc* d, int32_t* out_id) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!d) fail(FITB_ERR_ARG, "null plane-wave descriptor");
    if (d->waveform != FITB_WAVE_GAUSSIAN && d->waveform != FITB_WAVE_SINE)
        fail(FITB_ERR_ARG, "plane-wave waveform %d", d->waveform);
    if (d->waveform == FITB_WAVE_GAUSSIAN && !(d->den > 0.0)) fail(FITB_ERR_ARG, "gaussian plane wave needs den > 0");
    if (d->n_e < 0 || d->n_h < 0 || (d->n_e > 0 && (!d->e_idx || !d->e_coef || !d->e_delay)) ||
        (d->n_h > 0 && (!d->h_idx || !d->h_coef || !d->h_delay)))
        fail(FITB_ERR_ARG, "plane-wave patch arrays");
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "sources must be added before the first step");
    auto pw = std::make_unique<fitb::PlaneWaveHost>();
    // group the contributions of each entry, keeping their given order
    auto side = [&](bool is_h, int64_t n, const int64_t* idx, const double* coef, const double* delay,
                    fitb::DevBuf& off_b, fitb::DevBuf& start_b, fitb::DevBuf& coef_b, fitb::DevBuf& delay_b,
                    fitb::PlaneWaveSide& sd, std::vector<long long>* offs_out) {
        std::vector<long long> off((size_t)n);
        for (int64_t q = 0; q < n; ++q) off[(size_t)q] = H.flat_to_off(is_h, idx[q]);
        std::vector<int64_t> order((size_t)n);
        for (int64_t q = 0; q < n; ++q) order[(size_t)q] = q;
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return off[(size_t)a] < off[(size_t)b]; });
        std::vector<long long> uoff;
        std::vector<int> start;
        std::vector<double> c, dl;
        for (size_t r = 0; r < order.size(); ++r) {
            const int64_t q = order[r];
            if (r == 0 || off[(size_t)q] != uoff.back()) {
                uoff.push_back(off[(size_t)q]);
                start.push_back((int)c.size());
            }
            c.push_back(coef[q]);
            dl.push_back(delay[q]);
        }
        start.push_back((int)c.size());
        if (uoff.empty()) uoff.push_back(0);
        if (c.empty()) {
            c.push_back(0.0);
            dl.push_back(0.0);
        }
        fitb::upload(off_b, uoff);
        fitb::upload(start_b, start);
        fitb::upload(coef_b, c);
        fitb::upload(delay_b, dl);
        sd.n_unique = (long long)start.size() - 1;
        sd.off = off_b.as<long long>();
        sd.start = start_b.as<int>();
        sd.coef = coef_b.as<double>();
        sd.delay = delay_b.as<double>();
        if (offs_out) *offs_out = std::vector<long long>(uoff.begin(), uoff.begin() + sd.n_unique);
    };
    fitb::PlaneWaveDev& dv = pw->dev;
    side(false, d->n_e, d->e_idx, d->e_coef, d->e_delay, pw->e_off, pw->e_start, pw->e_coef, pw->e_delay, dv.e,
         &pw->e_off_host);
    side(true, d->n_h, d->h_idx, d->h_coef, d->h_delay, pw->h_off, pw->h_start, pw->h_coef, pw->h_delay, dv.h,
         nullptr);
    dv.waveform = d->waveform;
    dv.amplitude = d->amplitude;
    dv.t0 = d->t0;
    dv.den = d->den;
    dv.omega = d->omega;
    dv.dt = H.dt;
    pw->scale_host.assign((size_t)H.B, 1.0);
    fitb::upload(pw->scale, pw->scale_host);
    dv.scale = pw->scale.as<double>();
    H.pws.push_back(std::move(pw));
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    if (out_id) *out_id = (int32_t)H.pws.size() - 1;
    FITB_CATCH
}

int fitb_set_plane_wave_scale(fitb_handle* h, int32_t id, int32_t b, double scale) {
    FITB_TRY
    Handle& H = H_of(h);
    if (id < 0 || id >= (int32_t)H.pws.size()) fail(FITB_ERR_ARG, "plane wave %d out of range", id);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    auto& pw = *H.pws[(size_t)id];
    pw.scale_host[(size_t)b] = scale;
    ck(cudaMemcpyAsync(pw.scale.as<double>() + b, &pw.scale_host[(size_t)b], sizeof(double), cudaMemcpyHostToDevice,
                       H.stream),
       "plane-wave scale");
    ck(cudaStreamSynchronize(H.stream), "plane-wave scale sync");
    FITB_CATCH
}

int fitb_add_dft_monitor(fitb_handle* h, const fitb_dft_desc* d, int32_t* out_id) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!d || !d->freqs || !d->dx || !d->dy || !d->dz) fail(FITB_ERR_ARG, "null monitor argument");
    if (d->n_freq < 1) fail(FITB_ERR_ARG, "freqs must be a non-empty 1D array");
    if (d->stride < 1) fail(FITB_ERR_ARG, "stride must be >= 1");
    if (!(0 <= d->i0 && d->i0 < d->i1 && d->i1 <= H.g.nx && 0 <= d->j0 && d->j0 < d->j1 && d->j1 <= H.g.ny &&
          0 <= d->k0 && d->k0 < d->k1 && d->k1 <= H.g.nz))
        fail(FITB_ERR_ARG, "monitor box outside the grid");
    if ((d->comp_mask & 63) == 0) fail(FITB_ERR_ARG, "monitor records no component");
    if (H.steps_done != 0) fail(FITB_ERR_STATE, "monitors must be added before the first step");
    auto m = std::make_unique<fitb::DftHost>();
    fitb::DftDev& dv = m->dev;
    dv.i0 = d->i0;
    dv.j0 = d->j0;
    dv.k0 = d->k0;
    dv.ni = d->i1 - d->i0;
    dv.nj = d->j1 - d->j0;
    dv.nk = d->k1 - d->k0;
    dv.ncell = (long long)dv.ni * dv.nj * dv.nk;
    dv.ncomp = 0;
    for (int c = 0; c < 6; ++c)
        if (d->comp_mask & (1 << c)) dv.comps[dv.ncomp++] = c;
    dv.nf = d->n_freq;
    dv.stride = d->stride;
    dv.kahan = d->kahan ? 1 : 0;
    int K = (int)(49152 / (16 * (long long)dv.nf));
    dv.K = std::max(1, std::min(32, K));
    dv.dt = H.dt;
    std::vector<double> om((size_t)dv.nf);
    for (int f = 0; f < dv.nf; ++f) om[(size_t)f] = 2.0 * M_PI * d->freqs[f];
    fitb::upload(m->omega, om);
    int ld = std::max(H.g.nx, std::max(H.g.ny, H.g.nz)) + 1;
    dv.inv_ld = ld;
    std::vector<double> inv((size_t)(3 * ld), 1.0), dual((size_t)(3 * ld), 1.0);
    const double* ds[3] = {d->dx, d->dy, d->dz};
    const int ns[3] = {H.g.nx, H.g.ny, H.g.nz};
    for (int a = 0; a < 3; ++a) {
        const int n = ns[a];
        for (int q = 0; q < n; ++q) inv[(size_t)(a * ld + q)] = ds[a][q];
        // solver dual widths: boundary = full end cell (monitors/base.py:31-48)
        dual[(size_t)(a * ld)] = ds[a][0];
        for (int q = 1; q < n; ++q) dual[(size_t)(a * ld + q)] = 0.5 * (ds[a][q - 1] + ds[a][q]);
        dual[(size_t)(a * ld + n)] = ds[a][n - 1];
    }
    fitb::upload(m->inv, inv);
    fitb::upload(m->dual, dual);
    m->stage.alloc(sizeof(float) * (size_t)H.B * dv.K * dv.ncomp * dv.ncell);
    m->wst.alloc(sizeof(float2) * (size_t)dv.K * 2 * dv.nf);
    m->bins.alloc(sizeof(float2) * (size_t)H.B * dv.ncomp * dv.nf * dv.ncell);
    m->cmp.alloc(sizeof(float2) * (size_t)H.B * dv.ncomp * dv.nf * dv.ncell);
    m->base.alloc(sizeof(long long));
    dv.omega = m->omega.as<double>();
    dv.inv = m->inv.as<double>();
    dv.dual = m->dual.as<double>();
    dv.stage = m->stage.as<float>();
    dv.wst = m->wst.as<float2>();
    dv.bins = m->bins.as<float2>();
    dv.cmp = m->cmp.as<float2>();
    dv.base = m->base.as<long long>();
    m->i0 = d->i0; m->i1 = d->i1; m->j0 = d->j0; m->j1 = d->j1; m->k0 = d->k0; m->k1 = d->k1;
    if (out_id) *out_id = (int32_t)H.dft.size();
    H.dft.push_back(std::move(m));
    H.port_tables_dirty = true;
    fitb::invalidate_graphs(H);
    FITB_CATCH
}

int fitb_read_dft(fitb_handle* h, int32_t mon, int32_t b, int32_t comp, double* re, double* im, size_t count) {
    FITB_TRY
    Handle& H = H_of(h);
    if (mon < 0 || mon >= (int)H.dft.size()) fail(FITB_ERR_ARG, "monitor %d does not exist", mon);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    fitb::DftHost& m = *H.dft[mon];
    int ci = -1;
    for (int q = 0; q < m.dev.ncomp; ++q)
        if (m.dev.comps[q] == comp) ci = q;
    if (ci < 0) fail(FITB_ERR_ARG, "monitor %d does not record component %d", mon, comp);
    size_t n = (size_t)m.dev.nf * m.dev.ncell;
    if (count != n || !re || !im) fail(FITB_ERR_ARG, "expected %zu bins", n);
    fitb::dft_flush_pending(H);
    std::vector<float2> bins(n);
    size_t off = ((size_t)b * m.dev.ncomp + ci) * n;
    ck(cudaMemcpy(bins.data(), m.bins.as<float2>() + off, n * sizeof(float2), cudaMemcpyDeviceToHost), "read bins");
    for (size_t q = 0; q < n; ++q) {
        re[q] = bins[q].x;
        im[q] = bins[q].y;
    }
    FITB_CATCH
}

int fitb_step(fitb_handle* h, int64_t n_steps) {
    FITB_TRY
    Handle& H = H_of(h);
    fitb::run_steps(H, n_steps);
    ck(cudaGetLastError(), "step launch");
    FITB_CATCH
}

int fitb_step_timed(fitb_handle* h, int64_t n_steps, double* ms) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!ms) fail(FITB_ERR_ARG, "null argument");
    cudaEvent_t a, b;
    ck(cudaEventCreate(&a), "event");
    ck(cudaEventCreate(&b), "event");
    try {
        // prepare graphs / capacity outside the bracket
        fitb::run_steps(H, 0);
        ck(cudaEventRecord(a, H.stream), "event record");
        fitb::run_steps(H, n_steps);
        ck(cudaEventRecord(b, H.stream), "event record");
        ck(cudaEventSynchronize(b), "event sync");
        fitb::check_device_status(H);
        float f = 0.f;
        ck(cudaEventElapsedTime(&f, a, b), "elapsed");
        *ms = f;
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    FITB_CATCH
}

int fitb_time_stencil(fitb_handle* h, int32_t n_iter, double* ms_e, double* ms_h) {
    FITB_TRY
    Handle& H = H_of(h);
    fitb::check_ready(H);
    if (n_iter < 1 || !ms_e || !ms_h) fail(FITB_ERR_ARG, "bad argument");
    cudaEvent_t ev[3];
    for (auto& x : ev) ck(cudaEventCreate(&x), "event");
    if (H.stencil_mode == fitb::kModeFused) {
        // the whole E + H pass, alternating buffer sets; an even count
        // leaves the current set where it was
        fitb::refresh_port_tables(H);  // the slab form's unit lists
        const int n2 = 2 * ((n_iter + 1) / 2);
        ck(cudaEventRecord(ev[0], H.stream), "event record");
        int nl = 0;
        for (int q = 0; q < n2; ++q) {
            nl += fitb::launch_fused_any(H);
            H.cur ^= 1;
        }
        ck(cudaEventRecord(ev[1], H.stream), "event record");
        ck(cudaEventSynchronize(ev[1]), "event sync");
        H.launches += nl;
        fitb::check_device_status(H);
        float f1 = 0.f;
        ck(cudaEventElapsedTime(&f1, ev[0], ev[1]), "elapsed");
        for (auto& x : ev) cudaEventDestroy(x);
        *ms_e = f1 / n2;
        *ms_h = 0.0;
        return FITB_OK;
    }
    ck(cudaEventRecord(ev[0], H.stream), "event record");
    for (int q = 0; q < n_iter; ++q) fitb::launch_stencil_half(H, 0);
    ck(cudaEventRecord(ev[1], H.stream), "event record");
    for (int q = 0; q < n_iter; ++q) fitb::launch_stencil_half(H, 1);
    ck(cudaEventRecord(ev[2], H.stream), "event record");
    ck(cudaEventSynchronize(ev[2]), "event sync");
    fitb::check_device_status(H);
    H.launches += 2LL * n_iter;
    float f1 = 0.f, f2 = 0.f;
    ck(cudaEventElapsedTime(&f1, ev[0], ev[1]), "elapsed");
    ck(cudaEventElapsedTime(&f2, ev[1], ev[2]), "elapsed");
    for (auto& x : ev) cudaEventDestroy(x);
    *ms_e = f1 / n_iter;
    *ms_h = f2 / n_iter;
    FITB_CATCH
}

int fitb_sync(fitb_handle* h) {
    FITB_TRY
    Handle& H = H_of(h);
    ck(cudaStreamSynchronize(H.stream), "sync");
    fitb::check_device_status(H);
    FITB_CATCH
}

int fitb_probe_wait_timeout(fitb_handle* h, int32_t* status) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!status) fail(FITB_ERR_ARG, "null argument");
    ck(cudaStreamSynchronize(H.stream), "probe sync");
    ck(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream), "probe status reset");
    ck(fitb::launch_wait_probe(H.status.as<int>(), 1u << 16, H.stream), "wait probe launch");
    int st = 0;
    ck(cudaMemcpyAsync(&st, H.status.p, sizeof(int), cudaMemcpyDeviceToHost, H.stream), "probe status D2H");
    ck(cudaStreamSynchronize(H.stream), "probe sync");
    ck(cudaMemsetAsync(H.status.p, 0, sizeof(int), H.stream), "probe status reset");
    ck(cudaStreamSynchronize(H.stream), "probe sync");
    *status = st;
    FITB_CATCH
}

int fitb_mode_solve(int32_t device, int64_t n, const int64_t* rowptr, const int64_t* col, const double* val,
                    const double* m_diag, int32_t n_modes, double threshold, double* eigvals, double* eigvecs) {
    FITB_TRY
    if (n < 3 || n > 16384) fail(FITB_ERR_LIMIT, "mode problem of %lld unknowns (3 .. 16384)", (long long)n);
    if (n_modes < 1 || n_modes > 64 || n_modes > n - 2) fail(FITB_ERR_ARG, "n_modes %d", n_modes);
    if (!rowptr || !col || !val || !m_diag || !eigvals || !eigvecs) fail(FITB_ERR_ARG, "null argument");
    const long long nnz = rowptr[n];
    if (nnz < 0 || rowptr[0] != 0) fail(FITB_ERR_ARG, "row pointers");
    for (long long i = 0; i < n; ++i) {
        if (rowptr[i + 1] < rowptr[i]) fail(FITB_ERR_ARG, "row pointers not ascending");
        if (!(m_diag[i] > 0.0)) fail(FITB_ERR_ARG, "M diagonal entry %lld not positive", i);
    }
    for (long long q = 0; q < nnz; ++q)
        if (col[q] < 0 || col[q] >= n) fail(FITB_ERR_ARG, "column index %lld out of range", (long long)col[q]);
    ck(cudaSetDevice(device), "set device");
    fitb::DevBuf drp, dcol, dval, dm;
    fitb::upload(drp, std::vector<long long>(rowptr, rowptr + n + 1));
    fitb::upload(dcol, std::vector<long long>(col, col + nnz));
    fitb::upload(dval, std::vector<double>(val, val + nnz));
    fitb::upload(dm, std::vector<double>(m_diag, m_diag + n));
    cudaStream_t s;
    ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    const int rc = fitb::mode_eigensolve(n, drp.as<long long>(), dcol.as<long long>(), dval.as<double>(),
                                         dm.as<double>(), n_modes, threshold, eigvals, eigvecs, s);
    cudaStreamDestroy(s);
    if (rc == -3) fail(FITB_ERR_ARG, "fewer than %d eigenvalues above the threshold", n_modes);
    if (rc != 0) fail(FITB_ERR_CUDA, "mode eigensolve failed (%d)", rc);
    FITB_CATCH
}

int fitb_sparse_eigs(int32_t device, int64_t n, const int64_t* rowptr, const int64_t* col, const double* val,
                     int32_t n_null, const double* null_vecs, int32_t n_modes, double tol, double* eigvals,
                     double* eigvecs, double* residual, int32_t* iterations) {
    FITB_TRY
    if (n < 2 || n > (int64_t(1) << 26)) fail(FITB_ERR_LIMIT, "eigenproblem of %lld unknowns (2 .. 2^26)", (long long)n);
    if (n_modes < 1 || n_modes > 16) fail(FITB_ERR_LIMIT, "n_modes %d (1 .. 16)", n_modes);
    if (n_null < 0 || n_null > 8) fail(FITB_ERR_LIMIT, "n_null %d (0 .. 8)", n_null);
    if (n_modes + n_null > n) fail(FITB_ERR_ARG, "n_modes + n_null above n");
    if (!(tol > 0.0)) fail(FITB_ERR_ARG, "tolerance must be positive");
    if (!rowptr || !col || !val || !eigvals || !eigvecs || (n_null && !null_vecs)) fail(FITB_ERR_ARG, "null argument");
    const long long nnz = rowptr[n];
    if (nnz < 0 || nnz > (int64_t(1) << 30) || rowptr[0] != 0) fail(FITB_ERR_ARG, "row pointers");
    double bound = 0.0;
    for (long long i = 0; i < n; ++i) {
        if (rowptr[i + 1] < rowptr[i]) fail(FITB_ERR_ARG, "row pointers not ascending");
        double r = 0.0;
        for (long long q = rowptr[i]; q < rowptr[i + 1]; ++q) {
            if (col[q] < 0 || col[q] >= n) fail(FITB_ERR_ARG, "column index %lld out of range", (long long)col[q]);
            r += std::fabs(val[q]);
        }
        bound = std::max(bound, r);
    }
    if (!(bound > 0.0)) fail(FITB_ERR_ARG, "the matrix is zero");
    ck(cudaSetDevice(device), "set device");
    fitb::DevBuf drp, dcol, dval, dz;
    fitb::upload(drp, std::vector<long long>(rowptr, rowptr + n + 1));
    fitb::upload(dcol, std::vector<long long>(col, col + nnz));
    fitb::upload(dval, std::vector<double>(val, val + nnz));
    if (n_null) fitb::upload(dz, std::vector<double>(null_vecs, null_vecs + (size_t)n_null * n));
    cudaStream_t s;
    ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    double res = 0.0;
    int its = 0;
    const int rc = fitb::sparse_lowest_eigs(n, drp.as<long long>(), dcol.as<long long>(), dval.as<double>(), n_null,
                                            n_null ? dz.as<double>() : nullptr, n_modes, tol, 1.0001 * bound, eigvals,
                                            eigvecs, &res, &its, s);
    cudaStreamDestroy(s);
    if (residual) *residual = res;
    if (iterations) *iterations = its;
    if (rc == -4) fail(FITB_ERR_LIMIT, "not converged in %d iterations (residual %.3g of the spectral bound)", its, res);
    if (rc == -5) fail(FITB_ERR_ARG, "the start block lost its rank (fewer than n_modes + n_null independent vectors?)");
    if (rc != 0) fail(FITB_ERR_CUDA, "sparse eigensolve failed (%d)", rc);
    FITB_CATCH
}

int fitb_read_vi_async(fitb_handle* h, int32_t b, int64_t step0, int64_t n, double* V, double* I, int64_t* ticket) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!ticket) fail(FITB_ERR_ARG, "null ticket");
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    if (step0 < 0 || n < 0 || step0 + n > H.steps_done)
        fail(FITB_ERR_ARG, "steps [%lld, %lld) not issued", (long long)step0, (long long)(step0 + n));
    const size_t off = ((size_t)b * H.cap + step0) * H.nch;
    const size_t bytes = (size_t)n * H.nch * sizeof(double);
    if (H.nch > 0 && n > 0) {
        if (V) ck(cudaMemcpyAsync(V, H.recV.as<double>() + off, bytes, cudaMemcpyDeviceToHost, H.stream), "read V");
        if (I) ck(cudaMemcpyAsync(I, H.recI.as<double>() + off, bytes, cudaMemcpyDeviceToHost, H.stream), "read I");
    }
    const long long t = H.next_ticket++;
    ck(cudaEventRecord(H.tickets[t % Handle::kTickets], H.stream), "ticket record");
    *ticket = t;
    FITB_CATCH
}

int fitb_wait_ticket(fitb_handle* h, int64_t ticket) {
    FITB_TRY
    Handle& H = H_of(h);
    if (ticket < 0 || ticket >= H.next_ticket) fail(FITB_ERR_ARG, "ticket %lld was not issued", (long long)ticket);
    if (ticket < H.next_ticket - Handle::kTickets) {
        // its event has been reused: the work is older than a later ticket
        ck(cudaEventSynchronize(H.tickets[(H.next_ticket - Handle::kTickets) % Handle::kTickets]), "ticket wait");
    } else {
        ck(cudaEventSynchronize(H.tickets[ticket % Handle::kTickets]), "ticket wait");
    }
    FITB_CATCH
}

int fitb_query(fitb_handle* h, int32_t* done) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!done) fail(FITB_ERR_ARG, "null argument");
    const cudaError_t e = cudaStreamQuery(H.stream);
    if (e == cudaErrorNotReady) {
        *done = 0;
    } else {
        ck(e, "stream query");
        fitb::check_device_status(H);
        *done = 1;
    }
    FITB_CATCH
}

int fitb_steps_done(fitb_handle* h, int64_t* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!out) fail(FITB_ERR_ARG, "null argument");
    *out = H.steps_done;
    FITB_CATCH
}

int fitb_energy(fitb_handle* h, int32_t b, double* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (b < 0 || b >= H.B || !out) fail(FITB_ERR_ARG, "bad argument");
    if (H.prec == 4)
        fitb::energy_impl<float>(H, b, out);
    else
        fitb::energy_impl<double>(H, b, out);
    FITB_CATCH
}

int fitb_poll_signal_absmax(fitb_handle* h, int32_t b, double* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (b < 0 || b >= H.B || !out) fail(FITB_ERR_ARG, "bad argument");
    ck(cudaMemcpyAsync(out, H.absmax.as<double>() + b, sizeof(double), cudaMemcpyDeviceToHost, H.stream), "absmax");
    ck(cudaMemsetAsync(H.absmax.as<double>() + b, 0, sizeof(double), H.stream), "absmax reset");
    ck(cudaStreamSynchronize(H.stream), "absmax sync");
    FITB_CATCH
}

int fitb_channel_count(fitb_handle* h, int32_t* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!out) fail(FITB_ERR_ARG, "null argument");
    *out = H.nch;
    FITB_CATCH
}

int fitb_read_vi(fitb_handle* h, int32_t b, int64_t step0, int64_t n, double* V, double* I) {
    FITB_TRY
    Handle& H = H_of(h);
    if (b < 0 || b >= H.B) fail(FITB_ERR_ARG, "field set %d out of range", b);
    if (step0 < 0 || n < 0 || step0 + n > H.steps_done) fail(FITB_ERR_ARG, "steps [%lld, %lld) not recorded", (long long)step0, (long long)(step0 + n));
    if (H.nch == 0 || n == 0) return FITB_OK;
    // status word, V and I copied behind the steps on the handle's stream
    // into pinned memory, one synchronisation, then handed to the caller
    const size_t off = ((size_t)b * H.cap + step0) * H.nch;
    const size_t cnt = (size_t)n * H.nch, vb = cnt * sizeof(double);
    H.host_io.reserve(16 + 2 * vb);
    int* pst = static_cast<int*>(H.host_io.p);
    double* pv = reinterpret_cast<double*>(static_cast<char*>(H.host_io.p) + 16);
    double* pi = pv + cnt;
    const bool status = fitb::has_device_status(H);
    *pst = 0;
    if (status) ck(cudaMemcpyAsync(pst, H.status.p, sizeof(int), cudaMemcpyDeviceToHost, H.stream), "status D2H");
    if (V) ck(cudaMemcpyAsync(pv, H.recV.as<double>() + off, vb, cudaMemcpyDeviceToHost, H.stream), "read V");
    if (I) ck(cudaMemcpyAsync(pi, H.recI.as<double>() + off, vb, cudaMemcpyDeviceToHost, H.stream), "read I");
    ck(cudaStreamSynchronize(H.stream), "sync");
    if (status) fitb::raise_device_status(H, *pst);
    if (V) std::memcpy(V, pv, vb);
    if (I) std::memcpy(I, pi, vb);
    FITB_CATCH
}

int fitb_s_params(fitb_handle* h, int32_t nf, const double* f, const double* maps, const int32_t* icot,
                  const int32_t* excited, double a_threshold, double* S, double* A) {
    FITB_TRY
    Handle& H = H_of(h);
    if (nf < 1 || !f || !maps || !icot || !excited || !S) fail(FITB_ERR_ARG, "bad argument");
    if (H.nch == 0) fail(FITB_ERR_STATE, "no port channels are recorded");
    if (H.steps_done < 1) fail(FITB_ERR_STATE, "no steps recorded");
    for (int b = 0; b < H.B; ++b)
        if (excited[b] < -1 || excited[b] >= H.nch) fail(FITB_ERR_ARG, "excited channel %d out of range", excited[b]);
    ck(cudaStreamSynchronize(H.stream), "sync");
    fitb::check_device_status(H);
    const int nch = H.nch;
    fitb::DevBuf df, dmaps, dicot, dexc, xv, xi, dS, dA;
    fitb::upload(df, std::vector<double>(f, f + nf));
    fitb::upload(dmaps, std::vector<double>(maps, maps + (size_t)nch * 4 * nf * 2));
    fitb::upload(dicot, std::vector<int>(icot, icot + nch));
    fitb::upload(dexc, std::vector<int>(excited, excited + H.B));
    const size_t nx = (size_t)H.B * nch * nf;
    xv.alloc(nx * sizeof(double2), false);
    xi.alloc(nx * sizeof(double2), false);
    dS.alloc((size_t)nf * nch * H.B * sizeof(double2), false);
    if (A) dA.alloc((size_t)nf * H.B * sizeof(double2), false);
    fitb::launch_vi_dft(H.recV.as<double>(), H.recI.as<double>(), H.cap, nch, H.steps_done, H.B, df.as<double>(), nf,
                        H.dt, xv.as<double2>(), xi.as<double2>(), H.stream);
    fitb::launch_s_assemble(xv.as<double2>(), xi.as<double2>(), nch, nf, df.as<double>(), H.dt,
                            dmaps.as<double2>(), dicot.as<int>(), dexc.as<int>(), a_threshold, H.B,
                            dS.as<double2>(), A ? dA.as<double2>() : nullptr, H.stream);
    ck(cudaGetLastError(), "s-parameter launch");
    ck(cudaMemcpyAsync(S, dS.p, dS.bytes, cudaMemcpyDeviceToHost, H.stream), "S D2H");
    if (A) ck(cudaMemcpyAsync(A, dA.p, dA.bytes, cudaMemcpyDeviceToHost, H.stream), "A D2H");
    ck(cudaStreamSynchronize(H.stream), "S sync");
    H.launches += 2;
    FITB_CATCH
}

int fitb_state_size(fitb_handle* h, size_t* out) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!out) fail(FITB_ERR_ARG, "null argument");
    fitb::Writer w;
    if (H.prec == 4)
        fitb::write_state<float>(H, w);
    else
        fitb::write_state<double>(H, w);
    *out = w.n;
    FITB_CATCH
}

int fitb_state_export(fitb_handle* h, void* buf, size_t len) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!buf) fail(FITB_ERR_ARG, "null buffer");
    ck(cudaStreamSynchronize(H.stream), "sync");
    fitb::dft_flush_pending(H);
    std::vector<char> out;
    fitb::Writer w;
    w.out = &out;
    if (H.prec == 4)
        fitb::write_state<float>(H, w);
    else
        fitb::write_state<double>(H, w);
    if (out.size() != len) fail(FITB_ERR_ARG, "state buffer is %zu bytes, expected %zu", len, out.size());
    memcpy(buf, out.data(), out.size());
    FITB_CATCH
}

int fitb_state_import(fitb_handle* h, const void* buf, size_t len) {
    FITB_TRY
    Handle& H = H_of(h);
    if (!buf) fail(FITB_ERR_ARG, "null buffer");
    ck(cudaStreamSynchronize(H.stream), "sync");
    fitb::Reader r{(const char*)buf, len};
    if (H.prec == 4)
        fitb::read_state<float>(H, r);
    else
        fitb::read_state<double>(H, r);
    if (r.left != 0) fail(FITB_ERR_ARG, "state buffer has %zu trailing bytes", r.left);
    fitb::invalidate_graphs(H);
    H.port_tables_dirty = true;
    FITB_CATCH
}

}  // extern "C"
