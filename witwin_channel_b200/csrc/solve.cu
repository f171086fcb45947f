// Fused deterministic radiomap solve.
//
// Candidate preparation (per transmitter):
//   * reflection chains of coplanar groups per depth: exhaustive
//     (adjacent-distinct, paths.cu:364-406) when the reference's planning
//     guard allows it, otherwise discovered by tracing the FP64 Fibonacci
//     sphere (montecarlo.cu:713-731) with specular bounces and keeping the
//     unique group chains per depth (interactions/reflection.py:186-293,
//     541-569); FP64 image points are precomputed per chain;
//   * diffraction edges the source sees (exterior test + sampled-point
//     visibility prefilter, rayd/diffraction.cpp:380-403).
// Main kernel: one thread per (transmitter, receiver cell).  Each thread walks
// every candidate of its transmitter, traces the visibility segments through
// the BVH, evaluates the complex fields for every solve frequency and keeps
// the per-slot coherent sums in registers; each output cell is written once.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "em.cuh"
#include "internal.h"
#include "paths.cuh"
#include "solve.h"
#include "utd.cuh"
#include "kernels.cuh"

namespace wcb {

namespace {

constexpr int kBlock = 128;
constexpr int kMaxNF = 4;
constexpr long long kOrder1ExhaustiveLimit = 4096;      // interactions/reflection.py:30
constexpr long long kMultibounceExhaustiveLimit = 100000;  // interactions/reflection.py:31

// ------------------------------------------------------------ discovery
// Slot j of the discovery rays holds Fibonacci-lattice direction i = perm(j).
// The rays are split into bands of `band` consecutive indices (a Fibonacci
// number F_m near sqrt(32 pi count)); within a band the azimuth of index
// b0 + o is 2 pi frac(o / golden) up to a constant, whose order follows
// o * F_{m-1} mod F_m, so slot k of the band takes o = k * inv mod F_m (inv =
// F_{m-1}^-1 mod F_m).  A warp's 32 rays then leave in neighbouring
// directions and trace together; the tail band keeps the identity order.
// The chain tables depend only on the set of rays, not on their slots.
__global__ void k_fibonacci(int count, float* dirs, int band, int inv) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    long long i = j;
    if (band > 1) {
        const int b = j / band;
        if (b < count / band) i = (long long)b * band + ((long long)(j - b * band) * inv) % band;
    }
    const double golden = 1.618033988749894848204586834365638118;
    const double idx = double(i);
    const double az = idx / golden;
    const double az_u = az - floor(az);
    const double ev = count == 1 ? 0.0 : idx / double(count - 1);
    const double phi = 2.0 * kPi * az_u;
    const double z = 1.0 - 2.0 * ev;
    const double radial = sqrt(fmax(1.0 - z * z, 0.0));
    dirs[3 * j + 0] = float(radial * cos(phi));
    dirs[3 * j + 1] = float(radial * sin(phi));
    dirs[3 * j + 2] = float(z);
}

// Band size and multiplier of the coherent ray order for `count` rays (band
// 0: identity order).
static void fibonacci_bands(int count, int* band, int* inv) {
    *band = 0;
    *inv = 1;
    if (count < 256) return;
    const double target = std::sqrt(32.0 * kPi * double(count));
    long long prev = 1, cur = 2;
    while (cur < target) {
        const long long next = prev + cur;
        prev = cur;
        cur = next;
    }
    if (cur - target > target - prev) {  // the nearer Fibonacci number
        const long long p2 = cur - prev;
        cur = prev;
        prev = p2;
    }
    if (cur > count || cur < 2) return;
    // inverse of prev modulo cur (consecutive Fibonacci numbers are coprime)
    long long r0 = cur, r1 = prev, t0 = 0, t1 = 1;
    while (r1 != 0) {
        const long long q = r0 / r1;
        long long tmp = r0 - q * r1; r0 = r1; r1 = tmp;
        tmp = t0 - q * t1; t0 = t1; t1 = tmp;
    }
    if (r0 != 1) return;
    *band = int(cur);
    *inv = int(((t0 % cur) + cur) % cur);
}

template <typename G>
__global__ void __launch_bounds__(kBlock, sizeof(G) == 4 ? 8 : 4) k_discovery_trace(SceneDev sc, int count, int depth, const float* dirs,
                                                            const float* tx, int* groups_out, int* err,
                                                            unsigned long long* ray_counter) {
    extern __shared__ int stack[];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    V3<G> o = v3<G>(G(tx[0]), G(tx[1]), G(tx[2]));
    V3<G> d = v3<G>(G(dirs[3 * i]), G(dirs[3 * i + 1]), G(dirs[3 * i + 2]));
    int last = -1;
    bool alive = true;
    unsigned long long traced = 0;
    for (int k = 0; k < depth; ++k) {
        int hit_group = -1;
        if (alive) {
            ++traced;
            const G inf = sizeof(G) == 4 ? G(3e38) : G(1e300);
            Ray<G> r = make_ray<G>(o, d, G(1e-6), inf);
            Ignore ig = ignore_none();
            ig.f0 = last;
            G bt = inf;
            int bf = -1, bg = -1;
            traverse<1, G>(sc, r, ig, stack, err, &bt, &bf, &bg, NoSink{});
            if (bf >= 0) {
                hit_group = bg;
                const float* n = sc.face_normal + 3 * bf;
                const V3<G> nn = v3<G>(G(n[0]), G(n[1]), G(n[2]));
                o = o + d * bt;
                d = d - nn * (G(2) * dot(d, nn));
                last = bf;
            } else {
                alive = false;
            }
        }
        groups_out[size_t(i) * depth + k] = hit_group;
    }
    if (ray_counter) atomicAdd(ray_counter, traced);
}

// key for unique chains at depth k: (prefix rank << 21) | group
// Key (prefix rank, group) packed as pr << gbits | g, gbits = bits of the
// group count; rays without a hit at this depth get ~0 (sorted last: the sort
// covers key_bits() low bits, above every valid key).
__global__ void k_chain_keys(int count, int depth, int k, const int* groups, const int* prefix_rank, int gbits,
                             unsigned long long* keys, int* vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int g = groups[size_t(i) * depth + k];
    const int pr = k == 0 ? 0 : prefix_rank[i];
    unsigned long long key;
    if (g < 0 || pr < 0) key = ~0ull;
    else key = (static_cast<unsigned long long>(pr) << gbits) | static_cast<unsigned long long>(g);
    keys[i] = key;
    vals[i] = i;
}

__global__ void k_chain_flags(int count, const unsigned long long* keys, int* flags) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const bool valid = keys[i] != ~0ull;
    flags[i] = valid && (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// rank of each ray's chain after the inclusive scan of flags; the first ray
// of each run writes the chain's group ids into the chain table (when one is
// given) and the last valid element writes the chain count.
__global__ void k_chain_emit(int count, int depth, int k, const unsigned long long* keys, const int* vals,
                             const int* flags, const int* scan, const int* groups, int* rank_out, int* chain_groups,
                             int chain_cap, int* chain_count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int ray = vals[i];
    if (keys[i] == ~0ull) {
        rank_out[ray] = -1;
        return;
    }
    const int rank = scan[i] - 1;
    rank_out[ray] = rank;
    if (chain_groups != nullptr && flags[i] && rank < chain_cap) {
        for (int c = 0; c <= k; ++c) chain_groups[size_t(rank) * (k + 1) + c] = groups[size_t(ray) * depth + c];
    }
    if (chain_count != nullptr && (i == count - 1 || keys[i + 1] == ~0ull)) {
        *chain_count = min(rank + 1, chain_cap);
    }
}

// Bitmap form of the same dedup for small key spaces: bit (pr * G + g) is set
// for every ray's key; the unique keys in ascending order are the set bits in
// bit order, so a key's rank is the popcount of the bits below it (a scan of
// per-word popcounts plus the word's lower bits).  The ray that sets a bit
// writes that chain's groups (every ray with the key has the same group
// sequence), so the chain table equals the sorted form's.
__global__ void k_chain_bits(int count, int depth, int k, const int* groups, const int* prefix_rank, int G,
                             unsigned* bits, int* first) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int g = groups[size_t(i) * depth + k];
    const int pr = k == 0 ? 0 : prefix_rank[i];
    if (g < 0 || pr < 0) {
        first[i] = 0;
        return;
    }
    const long long key = (long long)pr * G + g;
    const unsigned bit = 1u << unsigned(key & 31);
    // one lane per distinct key of the warp (neighbouring rays share chains);
    // it reads the word first (bits are only ever set, so a set bit read here
    // is final) and takes the atomic only for a key not seen set
    const unsigned same = __match_any_sync(__activemask(), key);
    const int leader = __ffs(same) - 1;
    const int lane = threadIdx.x & 31;
    unsigned old = bit;
    if (lane == leader && !(__ldcg(bits + (key >> 5)) & bit)) old = atomicOr(bits + (key >> 5), bit);
    old = __shfl_sync(same, old, leader);
    first[i] = lane == leader && (old & bit) == 0u;
}

__global__ void k_word_popc(long long words, const unsigned* bits, int* out) {
    const long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (w < words) out[w] = __popc(bits[w]);
}

__global__ void k_chain_bits_emit(int count, int depth, int k, const int* groups, int* rank_io, int G,
                                  const unsigned* bits, const int* word_prefix, const int* first, int* chain_groups,
                                  int chain_cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int g = groups[size_t(i) * depth + k];
    const int pr = k == 0 ? 0 : rank_io[i];
    if (g < 0 || pr < 0) {
        rank_io[i] = -1;
        return;
    }
    const long long key = (long long)pr * G + g;
    const long long w = key >> 5;
    const int rank = word_prefix[w] + __popc(bits[w] & ((1u << unsigned(key & 31)) - 1u));
    rank_io[i] = rank;
    if (chain_groups != nullptr && first[i] && rank < chain_cap) {
        for (int c = 0; c <= k; ++c) chain_groups[size_t(rank) * (k + 1) + c] = groups[size_t(i) * depth + c];
    }
}

__global__ void k_chain_bits_count(long long words, const unsigned* bits, const int* word_prefix, int chain_cap,
                                   int* chain_count) {
    const int total = word_prefix[words - 1] + __popc(bits[words - 1]);
    *chain_count = min(total, chain_cap);
}

// exhaustive adjacent-distinct sequences (paths.cu:364-406)
__global__ void k_exhaustive_chains(long long total, int depth, int groups_n, int* chain_groups) {
    long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (row >= total) return;
    long long value = row;
    const long long base = depth > 1 ? groups_n - 1 : groups_n;
    long long div = 1;
    for (int p = 1; p < depth; ++p) div *= base;
    long long prev = -1;
    for (int col = 0; col < depth; ++col) {
        long long digit;
        if (depth > 1) {
            const long long raw = value / div;
            value -= raw * div;
            div = div > 1 ? div / base : 1;
            digit = col == 0 ? raw : (raw < prev ? raw : raw + 1);
            prev = digit;
        } else {
            digit = value;
        }
        chain_groups[row * depth + col] = int(digit);
    }
}

// FP64 images of the source through each chain's group planes.
__global__ void k_chain_images(SceneDev sc, const float* tx, int depth, const int* count_ptr, long long count_fixed,
                               const int* chain_groups, double* planes_out, double* images_out, float4* pre_out) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long count = count_ptr ? *count_ptr : count_fixed;
    if (c >= count) return;
    V3<double> p = v3<double>(tx[0], tx[1], tx[2]);
    for (int k = 0; k < depth; ++k) {
        const int g = chain_groups[c * depth + k];
        const double* pl = sc.group_plane + 4 * g;
        const V3<double> n = v3(pl[0], pl[1], pl[2]);
        p = p - n * (2.0 * (dot(p, n) - pl[3]));
        double* po = planes_out + (c * depth + k) * 4;
        po[0] = pl[0]; po[1] = pl[1]; po[2] = pl[2]; po[3] = pl[3];
        double* io = images_out + (c * depth + k) * 3;
        io[0] = p.x; io[1] = p.y; io[2] = p.z;
        if (k == depth - 1) {
            // FP32 copy of the last plane and image for the prefilter
            pre_out[2 * c] = make_float4(float(pl[0]), float(pl[1]), float(pl[2]), float(pl[3]));
            pre_out[2 * c + 1] = make_float4(float(p.x), float(p.y), float(p.z), __int_as_float(g));
        }
    }
}

// ------------------------------------------------------------ edge prefilter
template <typename G>
__global__ void __launch_bounds__(kBlock) k_edge_flags(SceneDev sc, const float* tx_pos, int t, double wavelength,
                                                       int* flags, int* err, unsigned long long* ray_counter) {
    // one warp per edge, one lane per sample point (at most 16): the edge is
    // Tx-visible when any sample is
    extern __shared__ int stack[];
    const long long gtid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int j = int(gtid >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= sc.num_edges) return;  // whole warps exit together
    const EdgeDev ed = sc.edges[j];
    const V3<double> S = v3<double>(tx_pos[3 * t], tx_pos[3 * t + 1], tx_pos[3 * t + 2]);
    const V3<double> c = v3(ed.pos[0], ed.pos[1], ed.pos[2]);
    const V3<double> e = v3(ed.dir[0], ed.dir[1], ed.dir[2]);
    V3<double> ds = S - c;
    ds = ds - e * dot(ds, e);
    const double phi_p = double(wedge_angle(ds, v3(ed.t0[0], ed.t0[1], ed.t0[2]), v3(ed.n0[0], ed.n0[1], ed.n0[2])));
    const bool exterior = phi_p <= ed.n * kPi;
    const double L = 2.0 * ed.half_length;
    int n = int(ceil(L / wavelength));
    n = n < 4 ? 4 : (n > 16 ? 16 : n);
    bool visible = false;
    if (exterior && lane < n) {
        Ignore ig = ignore_none();
        ig.f0 = ed.face0;
        ig.f1 = ed.face1;
        const V3<double> bis = v3(ed.bisector[0], ed.bisector[1], ed.bisector[2]);
        const double tt = -0.5 * L + (lane + 0.5) / n * L;
        const V3<double> p = c + e * tt + bis * kDiffractionRayBias;
        visible = !segment_blocked<G>(sc, cast3<G>(S), cast3<G>(p), ig, stack, err);
    }
    const unsigned any = __ballot_sync(0xffffffffu, visible);
    if (lane == 0) {
        flags[j] = any != 0u;
        if (ray_counter && exterior) atomicAdd(ray_counter, (unsigned long long)n);
    }
}

// ordered compaction of edge flags (one block per call)
__global__ void k_compact_flags(int n, const int* flags, int* list, int* count) {
    typedef cub::BlockScan<int, 256> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int start = 0; start < n; start += 256) {
        const int i = start + threadIdx.x;
        const int f = i < n ? flags[i] : 0;
        int pos, total;
        Scan(tmp).ExclusiveSum(f, pos, total);
        if (f) list[base + pos] = i;
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

// ------------------------------------------------------------ main kernel


// Start/end events of the four per-cell kernels (LoS+transmission,
// reflection, diffraction, finalize), each recorded on the kernel's stream.
struct ComponentEvents {
    cudaEvent_t start[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t end[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> vis;  // around each diffraction visibility launch
};

// Diffraction edge chunking: the visibility words of one chunk take at most
// kVisWordBudget 32-bit words (64 MiB), one word per (tile, edge).  The
// environment variable WCB_DIFFRACTION_CHUNK_WORDS lowers the budget (tests
// use it to run the multi-chunk path on small scenes).
constexpr long long kVisWordBudget = 16ll << 20;

static long long vis_word_budget() {
    const char* v = std::getenv("WCB_DIFFRACTION_CHUNK_WORDS");
    if (v != nullptr) {
        const long long n = std::atoll(v);
        if (n > 0 && n < kVisWordBudget) return n;
    }
    return kVisWordBudget;
}

struct DiffractionPlan {
    int chunk = 0;           // edges per chunk
    int chunks = 0;          // chunks covering the scene's edge count
    unsigned* words = nullptr;
    void* carry = nullptr;   // running per-cell sums between chunks (chunks > 1)
    bool run_vis = true;     // false when this frequency block reuses the words
};

static long long host_tiles_per_tx(const wcb_solve_desc& d) {
    if (d.rx_kind == 1) return (long long)((d.grid_rows + 7) / 8) * ((d.grid_cols + 3) / 4);
    return (d.num_rx + 31) / 32;
}

static DiffractionPlan diffraction_plan(const SceneDev& sc, const wcb_solve_desc& d) {
    DiffractionPlan dp;
    const long long tiles = host_tiles_per_tx(d) * d.num_tx;
    if (!(d.components & 4) || sc.num_edges <= 0 || tiles <= 0 || d.max_depth < 1) return dp;
    long long chunk = std::max(32ll, vis_word_budget() / tiles);
    chunk = std::min<long long>(chunk, sc.num_edges);
    dp.chunk = int(chunk);
    dp.chunks = int((sc.num_edges + chunk - 1) / chunk);
    return dp;
}

// LoS+transmission and diffraction go on `stream`, reflection on `side` (its
// candidate tables were built there); the caller joins the streams before
// the finalize kernel.
template <typename T, int NF>
void launch_nf(const MainParams& q0, unsigned blocks, int sdepth, size_t stack_bytes, cudaStream_t stream,
               cudaStream_t side, ComponentEvents* evs, const DiffractionPlan& dp) {
    const unsigned tiles = unsigned(tiles_per_tx(q0) * q0.num_tx);
    const size_t split_stack = size_t(sdepth) * kSplitBlock * 4;
    const int c = q0.components;
    MainParams q = q0;
    unsigned long long* rc = q0.ray_counter;
    if (c & 2) {
        if (evs) cudaEventRecord(evs->start[1], side);
        q.ray_counter = rc ? rc + 1 : nullptr;
        const size_t bytes = split_stack + kSplitWarps * sizeof(ReflShared<NF>) + size_t(kSplitWarps) * 32 * NF * 3 * 4;
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_reflect<T, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            attr = true;
        }
        k_reflect<T, NF><<<tiles, kSplitBlock, bytes, side>>>(q, sdepth);
        note_launch();
        if (evs) cudaEventRecord(evs->end[1], side);
    }
    if (evs) cudaEventRecord(evs->start[0], stream);
    if (c & (1 | 8)) {
        q.ray_counter = rc ? rc + 0 : nullptr;
        k_los_trans<T, NF><<<blocks, kCompBlock, stack_bytes, stream>>>(q);
        note_launch();
    }
    if (evs) cudaEventRecord(evs->end[0], stream);
    if (evs) cudaEventRecord(evs->start[2], stream);
    if ((c & 4) && dp.chunks > 0) {
        q.ray_counter = rc ? rc + 2 : nullptr;
        const size_t bytes = kSplitWarps * sizeof(DiffShared<NF>) + size_t(kSplitWarps) * 32 * NF * 9 * 4;
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_diffract_vis<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            cudaFuncSetAttribute(k_diffract_utd<T, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            attr = true;
        }
        for (int k = 0; k < dp.chunks; ++k) {
            const int j0 = k * dp.chunk;
            if (dp.run_vis) {
                std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
                if (evs) {
                    cudaEventCreate(&ev.first);
                    cudaEventCreate(&ev.second);
                    cudaEventRecord(ev.first, stream);
                }
                k_diffract_vis<T><<<tiles, kSplitBlock, split_stack, stream>>>(q, sdepth, j0, dp.chunk, dp.words);
                note_launch();
                if (evs) {
                    cudaEventRecord(ev.second, stream);
                    evs->vis.push_back(ev);
                }
            }
            k_diffract_utd<T, NF><<<tiles, kSplitBlock, bytes, stream>>>(q, j0, dp.chunk, dp.words,
                                                                        static_cast<T*>(dp.carry));
            note_launch();
        }
    }
    if (evs) cudaEventRecord(evs->end[2], stream);
}

template <typename T>
void launch_components(const MainParams& q, int nf, unsigned blocks, int sdepth, size_t stack_bytes, cudaStream_t stream,
                       cudaStream_t side, ComponentEvents* evs, const DiffractionPlan& dp) {
    switch (nf) {
        case 1: launch_nf<T, 1>(q, blocks, sdepth, stack_bytes, stream, side, evs, dp); break;
        case 2: launch_nf<T, 2>(q, blocks, sdepth, stack_bytes, stream, side, evs, dp); break;
        case 3: launch_nf<T, 3>(q, blocks, sdepth, stack_bytes, stream, side, evs, dp); break;
        default: launch_nf<T, 4>(q, blocks, sdepth, stack_bytes, stream, side, evs, dp); break;
    }
}

// One non-blocking side stream per device, created on first use.
cudaStream_t side_stream() {
    static std::mutex mu;
    static cudaStream_t streams[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (streams[dev] == nullptr) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    return streams[dev];
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

// ------------------------------------------------------------ host side
ProfileState& profile_state() {
    static ProfileState st;
    return st;
}

struct ChainPlan {
    bool exhaustive_o1;
    bool exhaustive_mb;
    long long cap[kMaxDepth];      // chains capacity per depth
    long long offset_int[kMaxDepth];
};

// Chain keys held in a bitmap when their space (prefix ranks x groups) is at
// most this many bits (8 MiB).  The environment variable
// WCB_CHAIN_BITMAP_BITS lowers the limit (0 keeps every depth on the sort;
// tests compare the two forms).
constexpr long long kChainBitmapBits = 1ll << 26;

static long long chain_bitmap_limit() {
    const char* v = std::getenv("WCB_CHAIN_BITMAP_BITS");
    if (v != nullptr) {
        const long long n = std::atoll(v);
        if (n >= 0 && n < kChainBitmapBits) return n;
    }
    return kChainBitmapBits;
}

// Size of the key space of depth k (0-based): the prefix chains at depth k-1
// number at most min(rays, G^k); 0 when it exceeds the bitmap limit.
static long long chain_key_bits(long long G, int rays, int k) {
    const long long limit = chain_bitmap_limit();
    if (G <= 0 || limit <= 0) return 0;
    long long prefixes = 1;
    for (int q = 0; q < k; ++q) {
        if (prefixes > (long long)rays / G + 1) { prefixes = rays; break; }
        prefixes = std::min<long long>(prefixes * G, rays);
    }
    if (prefixes > limit / G) return 0;
    return prefixes * G;
}

// bits needed to hold 0..n (n >= 0)
static int bit_width(long long n) {
    int b = 1;
    while (b < 63 && (n >> b) != 0) ++b;
    return b;
}

static long long seq_count(long long g, int d) {
    if (d > 1) {
        if (g <= 1) return 0;
        long long v = g;
        for (int i = 1; i < d; ++i) {
            if (v > LLONG_MAX / (g - 1)) return LLONG_MAX;
            v *= (g - 1);
        }
        return v;
    }
    return g;
}

// Per-transmitter chain offsets written on the device (no host staging, so a
// solve can be captured in a CUDA graph): offs[t*kMaxDepth + k] =
// t*per_tx + base[k].
struct ChainBase {
    long long v[kMaxDepth];
};

__global__ void k_chain_offsets(long long* offs, int num_tx, long long per_tx, ChainBase base) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num_tx * kMaxDepth) return;
    const int t = i / kMaxDepth, k = i - t * kMaxDepth;
    offs[i] = (long long)t * per_tx + base.v[k];
}

__global__ void k_set_count(int* dst, int value) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = value;
}

static ChainPlan make_plan(const SceneDev& sc, int max_depth, int rays) {
    ChainPlan pl;
    const long long G = sc.num_groups;
    pl.exhaustive_o1 = G <= kOrder1ExhaustiveLimit;
    pl.exhaustive_mb = true;
    for (int d = 2; d <= max_depth; ++d)
        if (seq_count(G, d) > kMultibounceExhaustiveLimit) pl.exhaustive_mb = false;
    long long off = 0;
    for (int d = 1; d <= kMaxDepth; ++d) {
        long long cap = 0;
        if (d <= max_depth) {
            if (d == 1) cap = pl.exhaustive_o1 ? G : rays;
            else cap = pl.exhaustive_mb ? seq_count(G, d) : rays;
        }
        pl.cap[d - 1] = cap;
        pl.offset_int[d - 1] = off;
        off += cap * d;
    }
    return pl;
}

struct WorkspaceLayout {
    size_t chain_counts, chain_offsets, chain_groups, chain_planes, chain_images, chain_pre;
    size_t disc_dirs, disc_groups, disc_keys, disc_keys2, disc_vals, disc_vals2, disc_flags, disc_scan, disc_rank,
        disc_temp, disc_bits, disc_word_count, disc_word_prefix;
    size_t disc_temp_bytes;
    size_t edge_flags, edge_list, edge_count;
    size_t diff_words, diff_carry;
    size_t overflow;
    size_t total;
    long long chain_ints_per_tx;
};

static WorkspaceLayout layout_for(const SceneDev& sc, const wcb_solve_desc& d, const ChainPlan& pl, int rays) {
    WorkspaceLayout L;
    const int T = d.num_tx;
    long long ints = 0;
    for (int k = 0; k < kMaxDepth; ++k) ints += pl.cap[k] * (k + 1);
    L.chain_ints_per_tx = ints;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = align_up(o + bytes); return at; };
    L.chain_counts = take(size_t(T) * kMaxDepth * 4);
    L.chain_offsets = take(size_t(T) * kMaxDepth * 8);
    L.chain_groups = take(size_t(T) * ints * 4);
    L.chain_planes = take(size_t(T) * ints * 4 * 8);
    L.chain_images = take(size_t(T) * ints * 3 * 8);
    L.chain_pre = take(size_t(T) * ints * 2 * 16);
    const bool disc = !(pl.exhaustive_o1 && pl.exhaustive_mb) && (d.components & 2);
    const size_t nr = disc ? size_t(rays) : 0;
    const int md = std::max(d.max_depth, 1);
    L.disc_dirs = take(nr * 3 * 4);
    L.disc_groups = take(nr * md * 4);
    L.disc_keys = take(nr * 8);
    L.disc_keys2 = take(nr * 8);
    L.disc_vals = take(nr * 4);
    L.disc_vals2 = take(nr * 4);
    L.disc_flags = take(nr * 4);
    L.disc_scan = take(nr * 4);
    L.disc_rank = take(nr * 4);
    // bitmap dedup: the largest key space any depth uses in that form
    long long max_bits = 0;
    if (nr)
        for (int k = 0; k < md; ++k) {
            const long long kb = chain_key_bits(sc.num_groups, int(nr), k);
            if (kb > 0) max_bits = std::max(max_bits, kb);
        }
    const size_t bm_words = size_t((max_bits + 31) / 32);
    L.disc_bits = take(bm_words * 4);
    L.disc_word_count = take(bm_words * 4);
    L.disc_word_prefix = take(bm_words * 4);
    size_t tb = 0;
    if (nr) {
        size_t a = 0, b = 0, c = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                        (int*)nullptr, (int*)nullptr, int(nr), 0, 64);
        cub::DeviceScan::InclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, int(nr));
        if (bm_words) cub::DeviceScan::ExclusiveSum(nullptr, c, (int*)nullptr, (int*)nullptr, int(bm_words));
        tb = std::max(a, std::max(b, c));
    }
    L.disc_temp_bytes = tb;
    L.disc_temp = take(tb);
    L.edge_flags = take(size_t(std::max(sc.num_edges, 1)) * 4);
    L.edge_list = take(size_t(T) * std::max(sc.num_edges, 1) * 4);
    L.edge_count = take(size_t(T) * 4);
    const DiffractionPlan dp = diffraction_plan(sc, d);
    const long long tiles = host_tiles_per_tx(d) * T;
    L.diff_words = take(dp.chunks > 0 ? size_t(tiles) * dp.chunk * 4 : 0);
    const long long cells = (long long)T * (d.rx_kind == 1 ? (long long)d.grid_rows * d.grid_cols : d.num_rx);
    L.diff_carry = take(dp.chunks > 1 ? size_t(cells) * kMaxNF * 9 * 8 : 0);
    L.overflow = take(64);
    L.total = o;
    return L;
}

int solve_workspace_size(const SceneHandle* h, const wcb_solve_desc* d, int64_t* bytes) {
    const int rays = d->discovery_rays > 0 ? d->discovery_rays : 262144;
    const ChainPlan pl = make_plan(h->dev, d->max_depth, rays);
    const WorkspaceLayout L = layout_for(h->dev, *d, pl, rays);
    *bytes = int64_t(L.total);
    return 0;
}

int solve(const SceneHandle* h, const wcb_solve_desc* d, const wcb_materials* m, const wcb_outputs* out, void* ws,
          int64_t ws_bytes, cudaStream_t stream) {
    // the scene record with this solve's traversal stack size: the BVH depth
    // bound, or the caller's smaller override (a descent that would push past
    // it drops the far subtree and sets status bit 0; no write leaves the stack)
    SceneDev sc = h->dev;
    if (d->stack_entries > 0) sc.stack_entries = std::min(std::max(d->stack_entries, 1), kStackDepth);
    if (d->num_tx < 0 || d->num_freq < 1 || d->max_depth < 0 || d->max_depth > kMaxDepth) return 1;
    const int rays = d->discovery_rays > 0 ? d->discovery_rays : 262144;
    const int T = d->num_tx;
    const int R = d->rx_kind == 1 ? d->grid_rows * d->grid_cols : d->num_rx;
    if (R < 0) return 1;
    const ChainPlan pl = make_plan(sc, d->max_depth, rays);
    const WorkspaceLayout L = layout_for(sc, *d, pl, rays);
    if (ws_bytes < int64_t(L.total)) return 3;
    char* base = static_cast<char*>(ws);
    int* chain_counts = reinterpret_cast<int*>(base + L.chain_counts);
    long long* chain_offsets = reinterpret_cast<long long*>(base + L.chain_offsets);
    int* chain_groups = reinterpret_cast<int*>(base + L.chain_groups);
    double* chain_planes = reinterpret_cast<double*>(base + L.chain_planes);
    double* chain_images = reinterpret_cast<double*>(base + L.chain_images);
    float4* chain_pre = reinterpret_cast<float4*>(base + L.chain_pre);
    int* edge_flags = reinterpret_cast<int*>(base + L.edge_flags);
    int* edge_list = reinterpret_cast<int*>(base + L.edge_list);
    int* edge_count = reinterpret_cast<int*>(base + L.edge_count);
    unsigned long long* overflow = reinterpret_cast<unsigned long long*>(base + L.overflow);
    unsigned long long* ray_counter = overflow + 1;       // preparation rays (discovery, edge prefilter)
    unsigned long long* main_ray_counter = overflow + 2;  // per-cell kernel rays: los+trans, reflection, diffraction
    const bool fp64 = d->precision == 1;
    ProfileState& prof = profile_state();
    cudaEvent_t ev_prep = nullptr, ev_main0 = nullptr, ev_main1 = nullptr;
    if (prof.enabled) {
        cudaEventCreate(&ev_prep);
        cudaEventCreate(&ev_main0);
        cudaEventCreate(&ev_main1);
        cudaEventRecord(ev_prep, stream);
        prof.main_ms = prof.prep_ms = 0.0;
        prof.rays = 0;
        prof.prep_rays = 0;
        prof.main_launches = 0;
    }
    if (T == 0 || R == 0) return 0;
    cudaMemsetAsync(chain_counts, 0, size_t(T) * kMaxDepth * 4, stream);
    cudaMemsetAsync(edge_count, 0, size_t(T) * 4, stream);
    cudaMemsetAsync(overflow, 0, 64, stream);
    if (out->status) cudaMemsetAsync(out->status, 0, 4, stream);
    if (out->row_count) cudaMemsetAsync(out->row_count, 0, 8, stream);
    if (out->transmission_overflow) cudaMemsetAsync(out->transmission_overflow, 0, 8, stream);
    // chain offsets (in chain-int units, per tx)
    std::vector<long long> offs(size_t(T) * kMaxDepth);
    std::vector<int> fixed_counts(size_t(T) * kMaxDepth, 0);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < kMaxDepth; ++k) offs[t * kMaxDepth + k] = t * L.chain_ints_per_tx + pl.offset_int[k];
    {
        ChainBase cb;
        for (int k = 0; k < kMaxDepth; ++k) cb.v[k] = pl.offset_int[k];
        const int n = T * kMaxDepth;
        k_chain_offsets<<<(n + 255) / 256, 256, 0, stream>>>(chain_offsets, T, L.chain_ints_per_tx, cb);
        note_launch();
    }
    const int B = 256;
    // traversal stacks: a descent pushes at most one entry per tree level, so
    // the measured BVH depth (+2) bounds them
    const size_t smem = size_t(sc.stack_entries) * kBlock * 4;
    int* err = out->status;
    // The reflection candidates (discovery, chain tables) and the reflection
    // kernel run on a side stream, overlapping the edge prefilter, the LoS and
    // the diffraction kernels on the caller's stream; the streams join before
    // the finalize kernel.
    cudaStream_t side = side_stream();
    if (side == nullptr) side = stream;
    cudaEvent_t fork = nullptr, join = nullptr;
    if (side != stream) {
        cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
        cudaEventRecord(fork, stream);
        cudaStreamWaitEvent(side, fork, 0);
    }
    // ---------------- reflection candidates
    if ((d->components & 2) && sc.num_faces > 0 && d->max_depth >= 1) {
        const bool need_disc = !(pl.exhaustive_o1 && (d->max_depth < 2 || pl.exhaustive_mb));
        float* dirs = reinterpret_cast<float*>(base + L.disc_dirs);
        if (need_disc) {
            int band = 0, inv = 1;
            fibonacci_bands(rays, &band, &inv);
            k_fibonacci<<<(rays + B - 1) / B, B, 0, side>>>(rays, dirs, band, inv);
            note_launch();
        }
        // exhaustive tables are identical for every tx: generate per tx
        for (int t = 0; t < T; ++t) {
            const float* txp = d->tx_pos + 3 * t;
            if (need_disc) {
                int* dg = reinterpret_cast<int*>(base + L.disc_groups);
                const int md = d->max_depth;
                if (fp64)
                    k_discovery_trace<double><<<(rays + kBlock - 1) / kBlock, kBlock, smem, side>>>(sc, rays, md, dirs, txp, dg, err, prof.enabled ? ray_counter : nullptr);
                else
                    k_discovery_trace<float><<<(rays + kBlock - 1) / kBlock, kBlock, smem, side>>>(sc, rays, md, dirs, txp, dg, err, prof.enabled ? ray_counter : nullptr);
                note_launch();
                const int gbits = bit_width(sc.num_groups);
                const int key_bits = std::min(64, gbits + bit_width(rays) + 1);
                unsigned long long* keys = reinterpret_cast<unsigned long long*>(base + L.disc_keys);
                unsigned long long* keys2 = reinterpret_cast<unsigned long long*>(base + L.disc_keys2);
                int* vals = reinterpret_cast<int*>(base + L.disc_vals);
                int* vals2 = reinterpret_cast<int*>(base + L.disc_vals2);
                int* flags = reinterpret_cast<int*>(base + L.disc_flags);
                int* scan = reinterpret_cast<int*>(base + L.disc_scan);
                int* rank = reinterpret_cast<int*>(base + L.disc_rank);
                void* temp = base + L.disc_temp;
                for (int k = 0; k < md; ++k) {
                    const int depth = k + 1;
                    const bool use_disc = depth == 1 ? !pl.exhaustive_o1 : !pl.exhaustive_mb;
                    // ranks are needed for the next depth even when this depth is exhaustive
                    int* cgrp = use_disc ? chain_groups + offs[t * kMaxDepth + k] : nullptr;
                    int* ccount = use_disc ? chain_counts + t * kMaxDepth + k : nullptr;
                    const long long kbits = chain_key_bits(sc.num_groups, rays, k);
                    if (kbits > 0) {
                        // small key space: bitmap dedup
                        const long long words = (kbits + 31) / 32;
                        unsigned* bits = reinterpret_cast<unsigned*>(base + L.disc_bits);
                        int* wpre = reinterpret_cast<int*>(base + L.disc_word_prefix);
                        int* wcnt = reinterpret_cast<int*>(base + L.disc_word_count);
                        cudaMemsetAsync(bits, 0, size_t(words) * 4, side);
                        k_chain_bits<<<(rays + B - 1) / B, B, 0, side>>>(rays, md, k, dg, rank, sc.num_groups, bits,
                                                                         flags);
                        k_word_popc<<<unsigned((words + B - 1) / B), B, 0, side>>>(words, bits, wcnt);
                        size_t tb = L.disc_temp_bytes;
                        cub::DeviceScan::ExclusiveSum(temp, tb, wcnt, wpre, int(words), side);
                        k_chain_bits_emit<<<(rays + B - 1) / B, B, 0, side>>>(rays, md, k, dg, rank, sc.num_groups,
                                                                              bits, wpre, flags, cgrp,
                                                                              use_disc ? int(pl.cap[k]) : 0);
                        if (ccount) k_chain_bits_count<<<1, 1, 0, side>>>(words, bits, wpre, int(pl.cap[k]), ccount);
                        note_launch(ccount ? 5 : 4);
                        continue;
                    }
                    k_chain_keys<<<(rays + B - 1) / B, B, 0, side>>>(rays, md, k, dg, rank, gbits, keys, vals);
                    size_t tb = L.disc_temp_bytes;
                    // only the key's used bits (+1 so the ~0 of a missing hit stays above)
                    cub::DeviceRadixSort::SortPairs(temp, tb, keys, keys2, vals, vals2, rays, 0, key_bits, side);
                    k_chain_flags<<<(rays + B - 1) / B, B, 0, side>>>(rays, keys2, flags);
                    tb = L.disc_temp_bytes;
                    cub::DeviceScan::InclusiveSum(temp, tb, flags, scan, rays, side);
                    k_chain_emit<<<(rays + B - 1) / B, B, 0, side>>>(rays, md, k, keys2, vals2, flags, scan, dg, rank,
                                                                       cgrp, use_disc ? int(pl.cap[k]) : 0, ccount);
                    note_launch(3);
                }
            }
            for (int k = 0; k < d->max_depth; ++k) {
                const int depth = k + 1;
                const bool exh = depth == 1 ? pl.exhaustive_o1 : pl.exhaustive_mb;
                int* cgrp = chain_groups + offs[t * kMaxDepth + k];
                double* cpl = chain_planes + offs[t * kMaxDepth + k] * 4;
                double* cim = chain_images + offs[t * kMaxDepth + k] * 3;
                float4* cpre = chain_pre + offs[t * kMaxDepth + k] * 2;
                if (exh) {
                    const long long total = pl.cap[k];
                    fixed_counts[t * kMaxDepth + k] = int(total);
                    if (total > 0) {
                        k_exhaustive_chains<<<int((total + B - 1) / B), B, 0, side>>>(total, depth, sc.num_groups, cgrp);
                        k_chain_images<<<int((total + B - 1) / B), B, 0, side>>>(sc, txp, depth, nullptr, total, cgrp, cpl, cim, cpre);
                        note_launch(2);
                    }
                    k_set_count<<<1, 32, 0, side>>>(chain_counts + t * kMaxDepth + k, int(total));
                    note_launch();
                } else {
                    const long long cap = pl.cap[k];
                    k_chain_images<<<int((cap + B - 1) / B), B, 0, side>>>(sc, txp, depth, chain_counts + t * kMaxDepth + k,
                                                                           0, cgrp, cpl, cim, cpre);
                    note_launch();
                }
            }
        }
    }
    // ---------------- diffraction edge prefilter
    if ((d->components & 4) && sc.num_edges > 0 && d->max_depth >= 1) {
        const double wavelength = kC0 / d->frequency_hz[0];
        for (int t = 0; t < T; ++t) {
            const long long threads = (long long)sc.num_edges * 32;
            const unsigned eblocks = unsigned((threads + kBlock - 1) / kBlock);
            if (fp64)
                k_edge_flags<double><<<eblocks, kBlock, smem, stream>>>(sc, d->tx_pos, t, wavelength, edge_flags, err, prof.enabled ? ray_counter : nullptr);
            else
                k_edge_flags<float><<<eblocks, kBlock, smem, stream>>>(sc, d->tx_pos, t, wavelength, edge_flags, err, prof.enabled ? ray_counter : nullptr);
            k_compact_flags<<<1, 256, 0, stream>>>(sc.num_edges, edge_flags, edge_list + size_t(t) * sc.num_edges, edge_count + t);
            note_launch(2);
        }
    }
    // ---------------- main kernel
    MainParams p;
    std::memset(&p, 0, sizeof(p));
    p.sc = sc;
    p.num_tx = T;
    p.num_rx = R;
    p.rx_kind = d->rx_kind;
    p.rx_pos = d->rx_pos;
    for (int k = 0; k < 3; ++k) {
        p.grid_origin[k] = d->grid_origin[k];
        p.grid_x[k] = d->grid_x_axis[k];
        p.grid_y[k] = d->grid_y_axis[k];
    }
    p.grid_rows = d->grid_rows;
    p.grid_cols = d->grid_cols;
    p.grid_spacing[0] = d->grid_spacing[0];
    p.grid_spacing[1] = d->grid_spacing[1];
    p.rx_pol = d->rx_pol;
    p.rx_pol_stride = d->rx_pol_stride;
    p.tx_pos = d->tx_pos;
    p.tx_power = d->tx_power;
    p.tx_pol = d->tx_pol;
    p.num_materials = m->num_materials;
    p.mat_eps_r = m->eps_r;
    p.mat_sigma_e = m->sigma_e;
    p.mat_mu_r = m->mu_r;
    p.mat_gain = m->gain;
    p.mat_thickness = m->thickness;
    p.mat_volumetric = m->volumetric;
    p.num_layers = m->num_layers;
    p.layer_offset = m->layer_offset;
    p.layer_count = m->layer_count;
    p.layer_thickness = m->layer_thickness;
    p.layer_eps_r = m->layer_eps_r;
    p.layer_sigma_e = m->layer_sigma_e;
    p.layer_mu_r = m->layer_mu_r;
    p.components = d->components;
    p.max_depth = d->max_depth;
    p.coherent = d->coherent;
    p.chain_count = chain_counts;
    p.chain_offset = chain_offsets;
    p.chain_groups = chain_groups;
    p.chain_planes = chain_planes;
    p.chain_images = chain_images;
    p.chain_pre = chain_pre;
    p.edge_count = edge_count;
    p.edge_list = edge_list;
    p.out_path_gain = out->path_gain;
    p.out_field = out->field;
    p.out_comp_power = out->comp_power;
    p.out_comp_field = out->comp_field;
    p.out_diff_vec_power = out->diff_vec_power;
    p.rows = static_cast<RowRec*>(out->rows);
    p.row_capacity = out->rows ? out->row_capacity : 0;
    p.row_counter = reinterpret_cast<unsigned long long*>(out->row_count);
    p.status = out->status;
    // transmission segments crossing more than max_depth walls: the caller's
    // counter when given (zeroed above), else the workspace's
    p.overflow_counter = out->transmission_overflow ? reinterpret_cast<unsigned long long*>(out->transmission_overflow)
                                                    : overflow;
    p.ray_counter = prof.enabled ? main_ray_counter : nullptr;
    p.num_freq_total = d->num_freq;
    const long long tiles = tiles_per_tx(p) * T;
    const long long blocks = (tiles + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const int sdepth = sc.stack_entries;
    const size_t stack_bytes = size_t(sdepth) * kCompBlock * 4;
    if (prof.enabled) cudaEventRecord(ev_main0, stream);
    ComponentEvents cev;
    double comp_ms[4] = {0, 0, 0, 0};
    double vis_ms = 0.0;
    DiffractionPlan dplan = diffraction_plan(sc, *d);
    dplan.words = reinterpret_cast<unsigned*>(base + L.diff_words);
    dplan.carry = dplan.chunks > 1 ? static_cast<void*>(base + L.diff_carry) : nullptr;
    if (prof.enabled)
        for (int i = 0; i < 4; ++i) {
            cudaEventCreate(&cev.start[i]);
            cudaEventCreate(&cev.end[i]);
        }
    for (int fb = 0; fb < d->num_freq; fb += kMaxNF) {
        const int nf = std::min(kMaxNF, d->num_freq - fb);
        p.freq_base = fb;
        for (int f = 0; f < nf; ++f) {
            p.freq[f] = d->frequency_hz[fb + f];
            p.k[f] = kTwoPi * p.freq[f] / kC0;
        }
        MainParams q = p;
        // material tables are addressed relative to this frequency chunk
        const long long mo = (long long)fb * m->num_materials;
        q.mat_eps_r = m->eps_r + mo;
        q.mat_sigma_e = m->sigma_e + mo;
        q.mat_mu_r = m->mu_r + mo;
        q.mat_gain = m->gain + mo;
        q.mat_thickness = m->thickness + mo;
        const long long lo = (long long)fb * m->num_layers;
        q.layer_thickness = m->layer_thickness ? m->layer_thickness + lo : nullptr;
        q.layer_eps_r = m->layer_eps_r ? m->layer_eps_r + lo : nullptr;
        q.layer_sigma_e = m->layer_sigma_e ? m->layer_sigma_e + lo : nullptr;
        q.layer_mu_r = m->layer_mu_r ? m->layer_mu_r + lo : nullptr;
        if (fb > 0) q.rows = nullptr;  // geometry rows are emitted once
        if (blocks <= 0) continue;
        ComponentEvents* evp = prof.enabled ? &cev : nullptr;
        // a single edge chunk keeps its visibility words for every frequency block
        dplan.run_vis = fb == 0 || dplan.chunks > 1;
        if (fp64) launch_components<double>(q, nf, unsigned(blocks), sdepth, stack_bytes, stream, side, evp, dplan);
        else launch_components<float>(q, nf, unsigned(blocks), sdepth, stack_bytes, stream, side, evp, dplan);
        if (side != stream) {
            cudaEventRecord(join, side);
            cudaStreamWaitEvent(stream, join, 0);
        }
        const long long nfin = (long long)T * R * nf;
        if (evp) cudaEventRecord(cev.start[3], stream);
        if (fp64) k_finalize<double><<<unsigned((nfin + 255) / 256), 256, 0, stream>>>(q, nf);
        else k_finalize<float><<<unsigned((nfin + 255) / 256), 256, 0, stream>>>(q, nf);
        note_launch();
        if (evp) {
            cudaEventRecord(cev.end[3], stream);
            cudaEventSynchronize(cev.end[3]);
            for (int i = 0; i < 4; ++i) {
                if (i == 1 && !(q.components & 2)) continue;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, cev.start[i], cev.end[i]);
                comp_ms[i] += ms;
            }
            for (auto& ev : cev.vis) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev.first, ev.second);
                vis_ms += ms;
                cudaEventDestroy(ev.first);
                cudaEventDestroy(ev.second);
            }
            cev.vis.clear();
        }
    }
    if (prof.enabled) {
        cudaEventRecord(ev_main1, stream);
        unsigned long long nr[4] = {0, 0, 0, 0};
        cudaMemcpyAsync(nr, ray_counter, 32, cudaMemcpyDeviceToHost, stream);
        int cc[kMaxDepth] = {0, 0, 0, 0, 0};
        int ec = 0;
        cudaMemcpyAsync(cc, chain_counts, sizeof(cc), cudaMemcpyDeviceToHost, stream);
        cudaMemcpyAsync(&ec, edge_count, 4, cudaMemcpyDeviceToHost, stream);
        cudaEventSynchronize(ev_main1);
        cudaStreamSynchronize(stream);
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev_prep, ev_main0);
        cudaEventElapsedTime(&b, ev_main0, ev_main1);
        prof.prep_ms = a;
        prof.main_ms = b;
        prof.prep_rays = (long long)nr[0];
        prof.rays = (long long)(nr[1] + nr[2] + nr[3]);
        prof.acc_rays += prof.rays + prof.prep_rays;
        for (int i = 0; i < 3; ++i) prof.kernel_rays[i] = (long long)nr[1 + i];
        for (int i = 0; i < 4; ++i) prof.kernel_ms[i] = comp_ms[i];
        prof.diffract_vis_ms = vis_ms;
        for (int i = 0; i < kMaxDepth; ++i) prof.chains[i] = cc[i];
        prof.edges = ec;
        for (int i = 0; i < 4; ++i) {
            cudaEventDestroy(cev.start[i]);
            cudaEventDestroy(cev.end[i]);
        }
        prof.main_launches = (d->num_freq + kMaxNF - 1) / kMaxNF;
        cudaEventDestroy(ev_prep);
        cudaEventDestroy(ev_main0);
        cudaEventDestroy(ev_main1);
    }
    if (side != stream) {
        // leave the side stream joined to the caller's stream (also when no
        // per-cell kernel ran)
        cudaEventRecord(join, side);
        cudaStreamWaitEvent(stream, join, 0);
        cudaEventDestroy(fork);
        cudaEventDestroy(join);
    }
    if (cudaGetLastError() != cudaSuccess) return 2;
    return 0;
}



}  // namespace wcb
