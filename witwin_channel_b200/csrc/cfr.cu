// Channel frequency response of path records: per (tx, rx) cell and
// subcarrier, H(f_k) = sum_p a_p exp(-j 2 pi (tau_p - tau_min) f_k)
// (the reference's PathResult.cfr, witwin/channel/path.py:646-656, with the
// delays normalised per link by their minimum; constants.py:51-53 for the
// narrowband law H(f_ref + df) = C exp(-j 2 pi df tau)).
//
// Two warps per link (cell): its records are a contiguous run of the canonical
// record list, located by one pass over the records.  Stores are coalesced
// and streaming, and each link's spectrum is written exactly once (zeros for a
// link without paths).  For a uniform grid f_k = f0 + k df each lane starts a
// path at its first subcarrier with the phase reduced in FP64 and advances it
// by a rotation; a non-uniform grid evaluates each phase directly (FP64
// reduction, FP32 sincos).
#include <cuda_runtime.h>

#include <climits>

#include "../../include/witwin_channel_b200.h"
#include "common.cuh"
#include "internal.h"

namespace wcb {
namespace {

constexpr int kCfrWarps = 8;

struct CfrParams {
    const int* tx;
    const int* rx;
    const float* delay;  // (K) seconds
    const float* field;  // (K,2) complex path coefficient
    long long count;
    int num_tx, num_rx;
    int num_freq;
    double f0, df;            // uniform grid (df != 0)
    const double* freqs;      // explicit grid (df == 0)
    int normalize;
    float* out;               // (T,R,NF) complex
};

// reduce 2 pi x (cycles) to [-pi, pi] in FP64 and return cos/sin in FP32; the
// argument is already reduced, so the hardware approximation (absolute error
// ~4e-7 on [-pi, pi]) is enough for the 1e-4 accuracy of the spectrum
WCB_D void cycles_sincos(double cycles, float* s, float* c) {
    const double frac = cycles - rint(cycles);
    __sincosf(float(kTwoPi * frac), s, c);
}

// [start, end) record range of every link from one pass over the canonical
// records (each link's records are contiguous); links without records keep
// the empty range the caller cleared to zero.
__global__ void k_link_ranges(long long n, const int* tx, const int* rx, int num_rx, int* start, int* end) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long cell = (long long)tx[i] * num_rx + rx[i];
    if (i == 0 || tx[i - 1] != tx[i] || rx[i - 1] != rx[i]) start[cell] = int(i);
    if (i == n - 1 || tx[i + 1] != tx[i] || rx[i + 1] != rx[i]) end[cell] = int(i + 1);
}

// Two warps per link: the 64 lanes of a link own subcarriers k = L + 64 m
// (L = lane within the link, m < M), so each warp store writes 32 consecutive
// complex values.  A lane computes its start phasor and the 64-subcarrier
// step once per path (FP64-reduced phase, FP32 sincos) and rotates through
// its M subcarriers; spectra longer than 64 M subcarriers take further passes.
constexpr int kLinkLanes = 64;
constexpr int kLinksPerBlock = kCfrWarps / 2;

template <bool UNIFORM, int M>
__global__ void __launch_bounds__(kCfrWarps * 32) k_cfr(CfrParams p, const int* link_start, const int* link_end) {
    const long long cell = blockIdx.x * (long long)kLinksPerBlock + (threadIdx.x >> 6);
    const int L = threadIdx.x & (kLinkLanes - 1);
    const int lane = threadIdx.x & 31;
    const long long cells = (long long)p.num_tx * p.num_rx;
    if (cell >= cells) return;  // both warps of a link leave together
    const int beg = link_start[cell], end = link_end[cell];
    double tau0 = 0.0;
    if (p.normalize && end > beg) {
        float mn = INFINITY;
        for (int q = beg + lane; q < end; q += 32) mn = fminf(mn, p.delay[q]);
        for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        tau0 = double(mn);
    }
    float2* o = reinterpret_cast<float2*>(p.out) + cell * p.num_freq;
    for (int base = 0; base < p.num_freq; base += kLinkLanes * M) {
        float acc_re[M], acc_im[M];
#pragma unroll
        for (int m = 0; m < M; ++m) { acc_re[m] = 0.f; acc_im[m] = 0.f; }
        const int k0 = base + L;
        for (int q = beg; q < end; ++q) {
            const double tau = double(p.delay[q]) - tau0;
            const float are = p.field[2 * q], aim = p.field[2 * q + 1];
            if (UNIFORM) {
                float s, c, ss, cs;
                cycles_sincos(-tau * (p.f0 + k0 * p.df), &s, &c);
                cycles_sincos(-tau * double(kLinkLanes) * p.df, &ss, &cs);
                float zr = c, zi = s;
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    acc_re[m] += are * zr - aim * zi;
                    acc_im[m] += are * zi + aim * zr;
                    const float nr = zr * cs - zi * ss;
                    zi = zr * ss + zi * cs;
                    zr = nr;
                }
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const int k = k0 + kLinkLanes * m;
                    if (k < p.num_freq) {
                        float s, c;
                        cycles_sincos(-tau * p.freqs[k], &s, &c);
                        acc_re[m] += are * c - aim * s;
                        acc_im[m] += are * s + aim * c;
                    }
                }
            }
        }
        // streaming stores: the spectrum is written once and not reread here
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const int k = k0 + kLinkLanes * m;
            if (k < p.num_freq) __stcs(o + k, make_float2(acc_re[m], acc_im[m]));
        }
    }
}

}  // namespace
}  // namespace wcb

extern "C" int wcb_cfr_workspace_size(int32_t num_tx, int32_t num_rx, int64_t* bytes) {
    if (bytes == nullptr || num_tx < 0 || num_rx < 0) return WCB_ERR_INVALID_ARGUMENT;
    *bytes = 2 * ((int64_t(num_tx) * num_rx * 4 + 255) / 256) * 256;
    return WCB_OK;
}

extern "C" int wcb_cfr(const int32_t* tx_id, const int32_t* rx_id, const float* delay_s, const float* path_field,
                       int64_t num_paths, int32_t num_tx, int32_t num_rx, int32_t num_freq, double f0, double df,
                       const double* frequencies, int32_t normalize_delays, float* out, void* workspace,
                       int64_t workspace_bytes, void* stream) {
    if (num_paths < 0 || num_paths > INT_MAX || num_tx < 0 || num_rx < 0 || out == nullptr)
        return WCB_ERR_INVALID_ARGUMENT;
    if (num_freq < 1) return WCB_ERR_INVALID_ARGUMENT;
    if (num_paths > 0 && (tx_id == nullptr || rx_id == nullptr || delay_s == nullptr || path_field == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    if (df == 0.0 && frequencies == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const long long cells = (long long)num_tx * num_rx;
    if (cells == 0) return WCB_OK;
    int64_t need = 0;
    wcb_cfr_workspace_size(num_tx, num_rx, &need);
    if (workspace == nullptr || workspace_bytes < need) return WCB_ERR_CAPACITY;
    int* link_start = static_cast<int*>(workspace);
    int* link_end = link_start + need / 8;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(workspace, 0, size_t(need), s);
    if (num_paths > 0) {
        wcb::k_link_ranges<<<unsigned((num_paths + 255) / 256), 256, 0, s>>>(num_paths, tx_id, rx_id, num_rx,
                                                                            link_start, link_end);
        wcb::note_launch();
    }
    wcb::CfrParams p;
    p.tx = tx_id;
    p.rx = rx_id;
    p.delay = delay_s;
    p.field = path_field;
    p.count = num_paths;
    p.num_tx = num_tx;
    p.num_rx = num_rx;
    p.num_freq = num_freq;
    p.f0 = f0;
    p.df = df;
    p.freqs = frequencies;
    p.normalize = normalize_delays != 0;
    p.out = out;
    const unsigned blocks = unsigned((cells + wcb::kLinksPerBlock - 1) / wcb::kLinksPerBlock);
    const unsigned th = wcb::kCfrWarps * 32;
    const int per_lane = (num_freq + wcb::kLinkLanes - 1) / wcb::kLinkLanes;
#define WCB_CFR_LAUNCH(M)                                                                  \
    if (df != 0.0) wcb::k_cfr<true, M><<<blocks, th, 0, s>>>(p, link_start, link_end);     \
    else wcb::k_cfr<false, M><<<blocks, th, 0, s>>>(p, link_start, link_end);
    if (per_lane <= 4) {
        WCB_CFR_LAUNCH(4)
    } else if (per_lane <= 8) {
        WCB_CFR_LAUNCH(8)
    } else {
        WCB_CFR_LAUNCH(16)
    }
#undef WCB_CFR_LAUNCH
    wcb::note_launch();
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}
