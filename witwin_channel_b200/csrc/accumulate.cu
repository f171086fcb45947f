// Flat per-cell accumulation of evaluated paths (the drop-in for the
// reference's deterministic_accumulate_flat op, native/channel/kernels/
// deterministic.cu:829-970 behind witwin/channel/kernels/deterministic.py:23-102).
//
// Each valid path adds (gain, field) to one of six slots of its (tx, rx)
// cell: 0 los, 1 reflection, 2 diffraction, 3 transmission (component 5),
// 4 scattering (6), 5 coupled (3, 4, 7).  The reference scatters with float
// atomics, so its sums have no fixed order; here the paths are stably sorted
// by output slot and each output is summed by one thread in path index order
// and written once, so results are reproducible bit for bit.  The
// finalisation follows the reference: coherent cells square the slot sums
// (scattering stays a power term unless scattering is coherent), incoherent
// cells add slot powers and report sqrt(power) as the field.  Every rounding
// is explicit (add, multiply, fused multiply-add, square root) so the FP32
// and FP64 results do not depend on compiler contraction; the coherent power
// is fma(re, re, im * im), which reproduces the reference's frozen outputs.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

#include "../../include/witwin_channel_b200.h"
#include "internal.h"

namespace wcb {
namespace {

constexpr int kSlots = 6;
constexpr int kScatteringSlot = 4;
constexpr int kBlock = 256;

__device__ __forceinline__ int accum_slot(int c) {
    if (c >= 0 && c < 3) return c;
    if (c == 3 || c == 4 || c == 7) return 5;
    if (c == 5) return 3;
    if (c == 6) return kScatteringSlot;
    return -1;
}

template <typename T>
struct Exact;
template <>
struct Exact<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
};
template <>
struct Exact<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
};

template <typename T>
__device__ __forceinline__ T cabs2_exact(T re, T im) {
    return Exact<T>::fma(re, re, Exact<T>::mul(im, im));
}

// key = slot * cells + cell, or slots * cells for a dropped path
__global__ void k_flat_keys(long long n, const unsigned char* valid, const int* tx, const int* rx, const int* cid,
                            int num_tx, int num_rx, unsigned long long* keys, int* idx) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long cells = (long long)num_tx * num_rx;
    const int s = accum_slot(cid[i]);
    const int t = tx[i], r = rx[i];
    const bool keep = valid[i] != 0 && s >= 0 && t >= 0 && r >= 0 && t < num_tx && r < num_rx;
    keys[i] = keep ? (unsigned long long)(s * cells + (long long)t * num_rx + r) : (unsigned long long)(kSlots * cells);
    idx[i] = int(i);
}

template <typename T>
__global__ void k_flat_sums(long long outputs, long long n, const unsigned long long* keys, const int* idx,
                            const T* gain, const T* re, const T* im, T* P, T* Re, T* Im) {
    const long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (o >= outputs) return;
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < (unsigned long long)o) lo = mid + 1;
        else hi = mid;
    }
    T p = T(0), a = T(0), b = T(0);
    for (long long q = lo; q < n && keys[q] == (unsigned long long)o; ++q) {
        const int i = idx[q];
        p = Exact<T>::add(p, gain[i]);
        a = Exact<T>::add(a, re[i]);
        b = Exact<T>::add(b, im[i]);
    }
    P[o] = p;
    Re[o] = a;
    Im[o] = b;
}

template <typename T>
__global__ void k_flat_finalize(long long cells, int coherent, int scattering_coherent, T* P, const T* Re,
                                const T* Im, T* power_total, T* field_real, T* field_imag) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= cells) return;
    T rs = T(0), is = T(0), ps = T(0), sp = T(0);
    for (int s = 0; s < kSlots; ++s) {
        const long long o = s * cells + c;
        const T re = Re[o], im = Im[o];
        if (coherent) {
            if (s == kScatteringSlot) {
                if (scattering_coherent) P[o] = cabs2_exact(re, im);
                sp = Exact<T>::add(sp, P[o]);
                continue;
            }
            P[o] = cabs2_exact(re, im);
        } else {
            if (s == kScatteringSlot && scattering_coherent) P[o] = cabs2_exact(re, im);
            ps = Exact<T>::add(ps, P[o]);
        }
        rs = Exact<T>::add(rs, re);
        is = Exact<T>::add(is, im);
    }
    if (coherent) {
        field_real[c] = rs;
        field_imag[c] = is;
        power_total[c] = Exact<T>::add(cabs2_exact(rs, is), sp);
    } else {
        power_total[c] = ps;
        field_real[c] = Exact<T>::sqrt(ps > T(0) ? ps : T(0));
        field_imag[c] = T(0);
    }
}

// Adjoint of the flat accumulation: one gather per path through the same
// slot/tx/rx gates, the |.|^2 and sqrt cell maps linearised at the saved
// forward outputs (d|z|^2 = 2 Re z dRe + 2 Im z dIm; d sqrt(P) = dP / 2 sqrt(P),
// zero at P <= 0).  Dropped paths get exact zeros.  Any cotangent may be null.
template <typename T>
struct FlatGrad {
    const T *cfr, *cfi, *ftr, *fti, *pt;          // saved forward outputs
    const T *g_pt, *g_ftr, *g_fti, *g_cp, *g_cfr, *g_cfi;
};

template <typename T>
__global__ void k_flat_backward(long long n, const unsigned char* valid, const int* tx, const int* rx, const int* cid,
                                int num_tx, int num_rx, int coherent, int scattering_coherent, FlatGrad<T> a,
                                T* grad_gain, T* grad_re, T* grad_im) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = accum_slot(cid[i]);
    const int t = tx[i], r = rx[i];
    T gg = T(0), gr = T(0), gi = T(0);
    if (valid[i] != 0 && s >= 0 && t >= 0 && r >= 0 && t < num_tx && r < num_rx) {
        const long long cells = (long long)num_tx * num_rx;
        const long long c = (long long)t * num_rx + r;
        const long long o = s * cells + c;
        if (a.g_cfr) gr += a.g_cfr[o];
        if (a.g_cfi) gi += a.g_cfi[o];
        const T half_inv_root = (a.pt && a.pt[c] > T(0)) ? T(1) / (T(2) * sqrt(a.pt[c])) : T(0);
        if (s == kScatteringSlot && scattering_coherent) {
            // |S|^2 reaches component_power, power_total and (incoherent) the sqrt pseudo-field
            T gp = T(0);
            if (a.g_cp) gp += a.g_cp[o];
            if (a.g_pt) gp += a.g_pt[c];
            if (!coherent && a.g_ftr) gp += a.g_ftr[c] * half_inv_root;
            gr += T(2) * a.cfr[o] * gp;
            gi += T(2) * a.cfi[o] * gp;
        } else if (coherent && s == kScatteringSlot) {
            if (a.g_cp) gg += a.g_cp[o];
            if (a.g_pt) gg += a.g_pt[c];
        } else if (coherent) {
            if (a.g_cp) {
                gr += T(2) * a.cfr[o] * a.g_cp[o];
                gi += T(2) * a.cfi[o] * a.g_cp[o];
            }
            if (a.g_ftr) gr += a.g_ftr[c];
            if (a.g_fti) gi += a.g_fti[c];
            if (a.g_pt) {
                gr += T(2) * a.ftr[c] * a.g_pt[c];
                gi += T(2) * a.fti[c] * a.g_pt[c];
            }
        } else {
            if (a.g_cp) gg += a.g_cp[o];
            if (a.g_pt) gg += a.g_pt[c];
            if (a.g_ftr) gg += a.g_ftr[c] * half_inv_root;
        }
    }
    grad_gain[i] = gg;
    grad_re[i] = gr;
    grad_im[i] = gi;
}

// Pushforward of the flat accumulation: the tangent slot sums (same ordered
// sums as the forward, over the tangent streams) linearised through the cell
// finalisation at the saved forward outputs.  On entry tP/tRe/tIm hold the
// tangent slot sums; tP is overwritten with the tangent component power.
template <typename T>
__global__ void k_flat_tangent_finalize(long long cells, int coherent, int scattering_coherent, const T* cfr,
                                        const T* cfi, const T* pt, T* tP, const T* tRe, const T* tIm, T* t_pt,
                                        T* t_ftr, T* t_fti) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= cells) return;
    T rs = T(0), is = T(0), fr = T(0), fi = T(0), tps = T(0), tsp = T(0);
    for (int s = 0; s < kSlots; ++s) {
        const long long o = s * cells + c;
        const T dre = tRe[o], dim = tIm[o];
        const bool field_power = (s == kScatteringSlot) ? scattering_coherent != 0 : coherent != 0;
        if (field_power) tP[o] = T(2) * (cfr[o] * dre + cfi[o] * dim);
        if (coherent && s == kScatteringSlot) {
            tsp += tP[o];
            continue;
        }
        tps += tP[o];
        rs += dre;
        is += dim;
        fr += cfr[o];
        fi += cfi[o];
    }
    if (coherent) {
        t_ftr[c] = rs;
        t_fti[c] = is;
        t_pt[c] = T(2) * (fr * rs + fi * is) + tsp;
    } else {
        t_pt[c] = tps;
        t_ftr[c] = pt[c] > T(0) ? tps / (T(2) * sqrt(pt[c])) : T(0);
        t_fti[c] = T(0);
    }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct FlatLayout {
    size_t keys, keys2, idx, idx2, tmp, tmp_bytes, total;
};

FlatLayout flat_layout(long long n) {
    FlatLayout L;
    const size_t m = size_t(std::max<long long>(n, 1));
    size_t o = 0;
    auto take = [&](size_t b) { const size_t a = o; o = align256(o + b); return a; };
    L.keys = take(m * 8);
    L.keys2 = take(m * 8);
    L.idx = take(m * 4);
    L.idx2 = take(m * 4);
    size_t a = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                    (int*)nullptr, (int*)nullptr, int(m), 0, 64);
    L.tmp_bytes = a;
    L.tmp = take(a);
    L.total = o;
    return L;
}

int end_bit_for(unsigned long long v) {
    int b = 1;
    while (b < 64 && (v >> b) != 0) ++b;
    return b;
}

template <typename T>
int accumulate_flat_t(const unsigned char* valid, const int* tx, const int* rx, const int* cid, const T* gain,
                      const T* re, const T* im, long long n, int num_tx, int num_rx, int coherent, int scat_coh,
                      T* power_total, T* field_real, T* field_imag, T* P, T* Re, T* Im, void* ws, long long ws_bytes,
                      cudaStream_t stream) {
    const long long cells = (long long)num_tx * num_rx;
    const long long outputs = kSlots * cells;
    if (cells == 0) return WCB_OK;
    const FlatLayout L = flat_layout(n);
    if (n > 0 && ws_bytes < (long long)L.total) return WCB_ERR_CAPACITY;
    unsigned long long* keys = nullptr;
    int* idx = nullptr;
    if (n > 0) {
        char* b = static_cast<char*>(ws);
        auto* k1 = reinterpret_cast<unsigned long long*>(b + L.keys);
        auto* k2 = reinterpret_cast<unsigned long long*>(b + L.keys2);
        int* i1 = reinterpret_cast<int*>(b + L.idx);
        int* i2 = reinterpret_cast<int*>(b + L.idx2);
        k_flat_keys<<<int((n + kBlock - 1) / kBlock), kBlock, 0, stream>>>(n, valid, tx, rx, cid, num_tx, num_rx, k1, i1);
        size_t tb = L.tmp_bytes;
        if (cub::DeviceRadixSort::SortPairs(b + L.tmp, tb, k1, k2, i1, i2, int(n), 0,
                                            end_bit_for((unsigned long long)outputs), stream) != cudaSuccess)
            return WCB_ERR_CUDA;
        note_launch(2);
        keys = k2;
        idx = i2;
    }
    k_flat_sums<T><<<int((outputs + kBlock - 1) / kBlock), kBlock, 0, stream>>>(outputs, n, keys, idx, gain, re, im, P,
                                                                                 Re, Im);
    k_flat_finalize<T><<<int((cells + kBlock - 1) / kBlock), kBlock, 0, stream>>>(cells, coherent, scat_coh, P, Re, Im,
                                                                                   power_total, field_real, field_imag);
    note_launch(2);
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}

template <typename T>
int accumulate_jvp_t(const unsigned char* valid, const int* tx, const int* rx, const int* cid, const T* t_gain,
                     const T* t_re, const T* t_im, long long n, int num_tx, int num_rx, int coherent, int scat_coh,
                     const wcb_accumulate_outputs* saved, const wcb_accumulate_outputs* tout, void* ws,
                     long long ws_bytes, cudaStream_t stream) {
    const long long cells = (long long)num_tx * num_rx;
    if (cells == 0) return WCB_OK;
    // tangent slot sums into the tangent component outputs (zeros stand in for absent streams)
    T* tP = static_cast<T*>(tout->component_power);
    T* tRe = static_cast<T*>(tout->component_field_real);
    T* tIm = static_cast<T*>(tout->component_field_imag);
    const FlatLayout L = flat_layout(n);
    if (n > 0 && ws_bytes < (long long)L.total + 3 * (long long)align256(size_t(n) * sizeof(T))) return WCB_ERR_CAPACITY;
    unsigned long long* keys = nullptr;
    int* idx = nullptr;
    const T *g = t_gain, *a = t_re, *b = t_im;
    if (n > 0) {
        char* base = static_cast<char*>(ws);
        char* zeros = base + L.total;
        const size_t zb = align256(size_t(n) * sizeof(T));
        if (!g) { cudaMemsetAsync(zeros, 0, zb, stream); g = reinterpret_cast<const T*>(zeros); }
        if (!a) { cudaMemsetAsync(zeros + zb, 0, zb, stream); a = reinterpret_cast<const T*>(zeros + zb); }
        if (!b) { cudaMemsetAsync(zeros + 2 * zb, 0, zb, stream); b = reinterpret_cast<const T*>(zeros + 2 * zb); }
        auto* k1 = reinterpret_cast<unsigned long long*>(base + L.keys);
        auto* k2 = reinterpret_cast<unsigned long long*>(base + L.keys2);
        int* i1 = reinterpret_cast<int*>(base + L.idx);
        int* i2 = reinterpret_cast<int*>(base + L.idx2);
        k_flat_keys<<<int((n + kBlock - 1) / kBlock), kBlock, 0, stream>>>(n, valid, tx, rx, cid, num_tx, num_rx, k1, i1);
        size_t tb = L.tmp_bytes;
        if (cub::DeviceRadixSort::SortPairs(base + L.tmp, tb, k1, k2, i1, i2, int(n), 0,
                                            end_bit_for((unsigned long long)(kSlots * cells)), stream) != cudaSuccess)
            return WCB_ERR_CUDA;
        note_launch(2);
        keys = k2;
        idx = i2;
    }
    const long long outputs = kSlots * cells;
    k_flat_sums<T><<<int((outputs + kBlock - 1) / kBlock), kBlock, 0, stream>>>(outputs, n, keys, idx, g, a, b, tP,
                                                                                 tRe, tIm);
    k_flat_tangent_finalize<T><<<int((cells + kBlock - 1) / kBlock), kBlock, 0, stream>>>(
        cells, coherent, scat_coh, static_cast<const T*>(saved->component_field_real),
        static_cast<const T*>(saved->component_field_imag), static_cast<const T*>(saved->power_total), tP, tRe, tIm,
        static_cast<T*>(tout->power_total), static_cast<T*>(tout->field_total_real),
        static_cast<T*>(tout->field_total_imag));
    note_launch(2);
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}

template <typename T>
int accumulate_backward_t(const unsigned char* valid, const int* tx, const int* rx, const int* cid, long long n,
                          int num_tx, int num_rx, int coherent, int scat_coh, const wcb_accumulate_outputs* saved,
                          const wcb_accumulate_outputs* grads, void* grad_gain, void* grad_re, void* grad_im,
                          cudaStream_t stream) {
    if (n == 0) return WCB_OK;
    FlatGrad<T> a;
    a.cfr = static_cast<const T*>(saved->component_field_real);
    a.cfi = static_cast<const T*>(saved->component_field_imag);
    a.ftr = static_cast<const T*>(saved->field_total_real);
    a.fti = static_cast<const T*>(saved->field_total_imag);
    a.pt = static_cast<const T*>(saved->power_total);
    a.g_pt = static_cast<const T*>(grads->power_total);
    a.g_ftr = static_cast<const T*>(grads->field_total_real);
    a.g_fti = static_cast<const T*>(grads->field_total_imag);
    a.g_cp = static_cast<const T*>(grads->component_power);
    a.g_cfr = static_cast<const T*>(grads->component_field_real);
    a.g_cfi = static_cast<const T*>(grads->component_field_imag);
    k_flat_backward<T><<<int((n + kBlock - 1) / kBlock), kBlock, 0, stream>>>(
        n, valid, tx, rx, cid, num_tx, num_rx, coherent, scat_coh, a, static_cast<T*>(grad_gain),
        static_cast<T*>(grad_re), static_cast<T*>(grad_im));
    note_launch();
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}

}  // namespace
}  // namespace wcb

extern "C" {

int wcb_accumulate_flat_jvp_workspace_size(int64_t num_paths, int32_t dtype, int64_t* bytes) {
    if (bytes == nullptr || num_paths < 0 || num_paths > INT_MAX - 1) return WCB_ERR_INVALID_ARGUMENT;
    if (dtype != WCB_DTYPE_F32 && dtype != WCB_DTYPE_F64) return WCB_ERR_INVALID_ARGUMENT;
    const size_t es = dtype == WCB_DTYPE_F32 ? 4 : 8;
    *bytes = num_paths == 0 ? 0
                            : int64_t(wcb::flat_layout(num_paths).total + 3 * wcb::align256(size_t(num_paths) * es));
    return WCB_OK;
}

int wcb_accumulate_flat_jvp(const uint8_t* valid, const int32_t* tx_id, const int32_t* rx_id,
                            const int32_t* component_id, const void* tangent_path_gain, const void* tangent_field_real,
                            const void* tangent_field_imag, int64_t num_paths, int32_t num_tx, int32_t num_rx,
                            int32_t coherent, int32_t scattering_coherent, int32_t dtype,
                            const wcb_accumulate_outputs* saved, const wcb_accumulate_outputs* tangent_out,
                            void* workspace, int64_t workspace_bytes, void* stream) {
    if (saved == nullptr || tangent_out == nullptr || num_paths < 0 || num_paths > INT_MAX - 1 || num_tx < 0 ||
        num_rx < 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (dtype != WCB_DTYPE_F32 && dtype != WCB_DTYPE_F64) return WCB_ERR_INVALID_ARGUMENT;
    if ((long long)num_tx * num_rx > 0 &&
        (tangent_out->power_total == nullptr || tangent_out->field_total_real == nullptr ||
         tangent_out->field_total_imag == nullptr || tangent_out->component_power == nullptr ||
         tangent_out->component_field_real == nullptr || tangent_out->component_field_imag == nullptr ||
         saved->component_field_real == nullptr || saved->component_field_imag == nullptr ||
         saved->power_total == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    if (num_paths > 0 && (valid == nullptr || tx_id == nullptr || rx_id == nullptr || component_id == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == WCB_DTYPE_F32)
        return wcb::accumulate_jvp_t<float>(valid, tx_id, rx_id, component_id,
                                            static_cast<const float*>(tangent_path_gain),
                                            static_cast<const float*>(tangent_field_real),
                                            static_cast<const float*>(tangent_field_imag), num_paths, num_tx, num_rx,
                                            coherent != 0, scattering_coherent != 0, saved, tangent_out, workspace,
                                            workspace_bytes, s);
    return wcb::accumulate_jvp_t<double>(valid, tx_id, rx_id, component_id,
                                         static_cast<const double*>(tangent_path_gain),
                                         static_cast<const double*>(tangent_field_real),
                                         static_cast<const double*>(tangent_field_imag), num_paths, num_tx, num_rx,
                                         coherent != 0, scattering_coherent != 0, saved, tangent_out, workspace,
                                         workspace_bytes, s);
}

int wcb_accumulate_flat_backward(const uint8_t* valid, const int32_t* tx_id, const int32_t* rx_id,
                                 const int32_t* component_id, int64_t num_paths, int32_t num_tx, int32_t num_rx,
                                 int32_t coherent, int32_t scattering_coherent, int32_t dtype,
                                 const wcb_accumulate_outputs* saved, const wcb_accumulate_outputs* grads,
                                 void* grad_path_gain, void* grad_field_real, void* grad_field_imag, void* stream) {
    if (saved == nullptr || grads == nullptr || num_paths < 0 || num_tx < 0 || num_rx < 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (dtype != WCB_DTYPE_F32 && dtype != WCB_DTYPE_F64) return WCB_ERR_INVALID_ARGUMENT;
    if (num_paths > 0 && (valid == nullptr || tx_id == nullptr || rx_id == nullptr || component_id == nullptr ||
                          grad_path_gain == nullptr || grad_field_real == nullptr || grad_field_imag == nullptr ||
                          saved->component_field_real == nullptr || saved->component_field_imag == nullptr ||
                          saved->field_total_real == nullptr || saved->field_total_imag == nullptr ||
                          saved->power_total == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == WCB_DTYPE_F32)
        return wcb::accumulate_backward_t<float>(valid, tx_id, rx_id, component_id, num_paths, num_tx, num_rx,
                                                 coherent != 0, scattering_coherent != 0, saved, grads, grad_path_gain,
                                                 grad_field_real, grad_field_imag, s);
    return wcb::accumulate_backward_t<double>(valid, tx_id, rx_id, component_id, num_paths, num_tx, num_rx,
                                              coherent != 0, scattering_coherent != 0, saved, grads, grad_path_gain,
                                              grad_field_real, grad_field_imag, s);
}

int wcb_accumulate_flat_workspace_size(int64_t num_paths, int64_t* bytes) {
    if (bytes == nullptr || num_paths < 0 || num_paths > INT_MAX - 1) return WCB_ERR_INVALID_ARGUMENT;
    *bytes = num_paths == 0 ? 0 : int64_t(wcb::flat_layout(num_paths).total);
    return WCB_OK;
}

int wcb_accumulate_flat(const uint8_t* valid, const int32_t* tx_id, const int32_t* rx_id, const int32_t* component_id,
                        const void* path_gain, const void* field_real, const void* field_imag, int64_t num_paths,
                        int32_t num_tx, int32_t num_rx, int32_t coherent, int32_t scattering_coherent, int32_t dtype,
                        const wcb_accumulate_outputs* out, void* workspace, int64_t workspace_bytes, void* stream) {
    if (out == nullptr || num_paths < 0 || num_paths > INT_MAX - 1 || num_tx < 0 || num_rx < 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (dtype != WCB_DTYPE_F32 && dtype != WCB_DTYPE_F64) return WCB_ERR_INVALID_ARGUMENT;
    if ((long long)num_tx * num_rx * 6 >= (1ll << 62)) return WCB_ERR_INVALID_ARGUMENT;
    if ((long long)num_tx * num_rx > 0 &&
        (out->power_total == nullptr || out->field_total_real == nullptr || out->field_total_imag == nullptr ||
         out->component_power == nullptr || out->component_field_real == nullptr ||
         out->component_field_imag == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    if (num_paths > 0 && (valid == nullptr || tx_id == nullptr || rx_id == nullptr || component_id == nullptr ||
                          path_gain == nullptr || field_real == nullptr || field_imag == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == WCB_DTYPE_F32)
        return wcb::accumulate_flat_t<float>(
            valid, tx_id, rx_id, component_id, static_cast<const float*>(path_gain),
            static_cast<const float*>(field_real), static_cast<const float*>(field_imag), num_paths, num_tx, num_rx,
            coherent != 0, scattering_coherent != 0, static_cast<float*>(out->power_total),
            static_cast<float*>(out->field_total_real), static_cast<float*>(out->field_total_imag),
            static_cast<float*>(out->component_power), static_cast<float*>(out->component_field_real),
            static_cast<float*>(out->component_field_imag), workspace, workspace_bytes, s);
    return wcb::accumulate_flat_t<double>(
        valid, tx_id, rx_id, component_id, static_cast<const double*>(path_gain),
        static_cast<const double*>(field_real), static_cast<const double*>(field_imag), num_paths, num_tx, num_rx,
        coherent != 0, scattering_coherent != 0, static_cast<double*>(out->power_total),
        static_cast<double*>(out->field_total_real), static_cast<double*>(out->field_total_imag),
        static_cast<double*>(out->component_power), static_cast<double*>(out->component_field_real),
        static_cast<double*>(out->component_field_imag), workspace, workspace_bytes, s);
}

}  // extern "C"
