// Channel frequency response of path records: per (tx, rx) cell and
// subcarrier, H(f_k) = sum_p a_p exp(-j 2 pi (tau_p - tau_min) f_k)
// (the reference's PathResult.cfr, witwin/channel/path.py:646-656, with the
// delays normalised per link by their minimum; constants.py:51-53 for the
// narrowband law H(f_ref + df) = C exp(-j 2 pi df tau)).
//
// One warp per cell: the cell's records are a contiguous run of the
// canonical (rx, tx)-sorted record list, found by binary search.  Lane l owns
// subcarriers k = l + 32 m, so every store of the warp writes 32 consecutive
// complex values (256 B, coalesced) and each cell's spectrum is written
// exactly once (zeros for a cell without paths).  For a uniform subcarrier
// grid f_k = f0 + k df a lane starts each path at its first subcarrier with
// the phase reduced in FP64 and advances it by the rotation
// exp(-j 2 pi tau 32 df), renormalised every 16 steps; a non-uniform grid
// evaluates each phase directly (FP64 reduction, FP32 sincos).
#include <cuda_runtime.h>

#include <climits>

#include "../../include/witwin_channel_b200.h"
#include "common.cuh"
#include "internal.h"

namespace wcb {
namespace {

constexpr int kCfrWarps = 8;
constexpr int kMaxLaneSubcarriers = 64;  // K <= 2048

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

// reduce 2 pi x (cycles) to [-pi, pi) in FP64 and return cos/sin in FP32
WCB_D void cycles_sincos(double cycles, float* s, float* c) {
    const double frac = cycles - rint(cycles);
    sincosf(float(kTwoPi * frac), s, c);
}

// M = subcarriers per lane (K <= 32 M), a compile-time bound so the
// accumulators stay in registers
template <bool UNIFORM, int M>
__global__ void __launch_bounds__(kCfrWarps * 32) k_cfr(CfrParams p) {
    const long long cell = blockIdx.x * (long long)kCfrWarps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const long long cells = (long long)p.num_tx * p.num_rx;
    if (cell >= cells) return;
    const int t = int(cell / p.num_rx);
    const int r = int(cell - (long long)t * p.num_rx);
    // records sorted by (rx, tx): lower bound of (r, t)
    long long lo = 0, hi = p.count;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        const int mr = p.rx[mid], mt = p.tx[mid];
        if (mr < r || (mr == r && mt < t)) lo = mid + 1;
        else hi = mid;
    }
    long long end = lo;
    while (end < p.count && p.rx[end] == r && p.tx[end] == t) ++end;
    double tau0 = 0.0;
    if (p.normalize && end > lo) {
        float m = INFINITY;
        for (long long q = lo + lane; q < end; q += 32) m = fminf(m, p.delay[q]);
        for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
        tau0 = double(m);
    }
    const int per_lane = (p.num_freq + 31) / 32;
    float acc_re[M], acc_im[M];
#pragma unroll
    for (int m = 0; m < M; ++m) { acc_re[m] = 0.f; acc_im[m] = 0.f; }
    for (long long q = lo; q < end; ++q) {
        const double tau = double(p.delay[q]) - tau0;
        const float are = p.field[2 * q], aim = p.field[2 * q + 1];
        if (UNIFORM) {
            // phase of subcarrier k: -2 pi tau (f0 + k df); lane's first k = lane
            float s, c, ss, cs;
            cycles_sincos(-tau * (p.f0 + lane * p.df), &s, &c);
            cycles_sincos(-tau * 32.0 * p.df, &ss, &cs);
            float zr = c, zi = s;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (m < per_lane) {
                    acc_re[m] += are * zr - aim * zi;
                    acc_im[m] += are * zi + aim * zr;
                    const float nr = zr * cs - zi * ss;
                    const float ni = zr * ss + zi * cs;
                    zr = nr;
                    zi = ni;
                    if ((m & 15) == 15) {  // keep |z| = 1 over long runs
                        const float inv = rsqrtf(zr * zr + zi * zi);
                        zr *= inv;
                        zi *= inv;
                    }
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const int k = lane + 32 * m;
                if (m < per_lane && k < p.num_freq) {
                    float s, c;
                    cycles_sincos(-tau * p.freqs[k], &s, &c);
                    acc_re[m] += are * c - aim * s;
                    acc_im[m] += are * s + aim * c;
                }
            }
        }
    }
    float2* o = reinterpret_cast<float2*>(p.out) + cell * p.num_freq;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const int k = lane + 32 * m;
        if (m < per_lane && k < p.num_freq) o[k] = make_float2(acc_re[m], acc_im[m]);
    }
}

}  // namespace
}  // namespace wcb

extern "C" int wcb_cfr(const int32_t* tx_id, const int32_t* rx_id, const float* delay_s, const float* path_field,
                       int64_t num_paths, int32_t num_tx, int32_t num_rx, int32_t num_freq, double f0, double df,
                       const double* frequencies, int32_t normalize_delays, float* out, void* stream) {
    if (num_paths < 0 || num_tx < 0 || num_rx < 0 || out == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    if (num_freq < 1 || num_freq > 32 * wcb::kMaxLaneSubcarriers) return WCB_ERR_NOT_SUPPORTED;
    if (num_paths > 0 && (tx_id == nullptr || rx_id == nullptr || delay_s == nullptr || path_field == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    if (df == 0.0 && frequencies == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const long long cells = (long long)num_tx * num_rx;
    if (cells == 0) return WCB_OK;
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
    const unsigned blocks = unsigned((cells + wcb::kCfrWarps - 1) / wcb::kCfrWarps);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int per_lane = (num_freq + 31) / 32;
    const unsigned th = wcb::kCfrWarps * 32;
#define WCB_CFR_LAUNCH(M)                                                      \
    if (df != 0.0) wcb::k_cfr<true, M><<<blocks, th, 0, s>>>(p);               \
    else wcb::k_cfr<false, M><<<blocks, th, 0, s>>>(p);
    if (per_lane <= 4) {
        WCB_CFR_LAUNCH(4)
    } else if (per_lane <= 16) {
        WCB_CFR_LAUNCH(16)
    } else if (per_lane <= 32) {
        WCB_CFR_LAUNCH(32)
    } else {
        WCB_CFR_LAUNCH(64)
    }
#undef WCB_CFR_LAUNCH
    wcb::note_launch();
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}
