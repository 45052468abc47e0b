// Orion commit on the device: expander encode (gathers over target-sorted
// graphs) and the SHA-256 Merkle tree. See orion.h for the layout.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "fp2.cuh"
#include "glibc_rand.h"
#include "orion.h"
#include "runtime.h"
#include "sha256.cuh"

namespace tp {
namespace orion {

namespace {

thread_local int g_launches = 0;
std::atomic<int> g_leaf_chunks{1};   // launches the row-leaf chains are split into
std::atomic<int> g_gather_cpl{2};    // columns per lane of the 61 x 31-bit gathers of large graphs

// kernel-timer tags (runtime.h timer_*): commit kernels are 9100 + kind
constexpr int kTagLoad = 9100, kTagGatherBytes = 9101, kTagGather = 9102, kTagLeaf = 9103, kTagTree = 9104;

long long c_targets(long long n) { return (long long)(0.238 * (double)n); }
long long d_targets(long long n, long long L) { return (long long)((double)n * (1.72 - 1) - (double)L); }

// encode_output_len (linear_code_encode.h:8-15) with D[dep].R from expander_init
long long cw_len_rec(long long n)
{
    if (n <= kThreshold) return n;
    const long long L = cw_len_rec(c_targets(n));
    return n + L + d_targets(n, L);
}

struct HostGraph {
    long long L, R;
    std::vector<unsigned> ptr;       // R + 1
    std::vector<unsigned> src;       // edges, grouped by target
    std::vector<ulonglong2> w;
};

// generate_random_expander (expanders.h:19-45): for each source i, d draws of
// (target = rand() % R, weight = (real rand() % p, img rand() % p)); stored by target
HostGraph gen_graph(GlibcRand& g, long long L, long long R, int d)
{
    HostGraph h;
    h.L = L;
    h.R = R;
    std::vector<unsigned> tgt((size_t)(L * d));
    std::vector<ulonglong2> wt((size_t)(L * d));
    std::vector<unsigned> cnt((size_t)R + 1, 0);
    for (long long i = 0; i < L; ++i)
        for (int j = 0; j < d; ++j) {
            const long long t = (long long)g.next() % R;
            const uint64_t re = (uint64_t)g.next() % P61;
            const uint64_t im = (uint64_t)g.next() % P61;
            tgt[(size_t)(i * d + j)] = (unsigned)t;
            wt[(size_t)(i * d + j)] = make_ulonglong2(im, re);
            cnt[(size_t)t + 1]++;
        }
    h.ptr.assign((size_t)R + 1, 0);
    for (long long t = 0; t < R; ++t) h.ptr[(size_t)t + 1] = h.ptr[(size_t)t] + cnt[(size_t)t + 1];
    h.src.resize((size_t)(L * d));
    h.w.resize((size_t)(L * d));
    std::vector<unsigned> fill(h.ptr.begin(), h.ptr.end() - 1);
    for (long long i = 0; i < L; ++i)
        for (int j = 0; j < d; ++j) {
            const unsigned t = tgt[(size_t)(i * d + j)];
            const unsigned e = fill[t]++;
            h.src[e] = (unsigned)i;
            h.w[e] = wt[(size_t)(i * d + j)];
        }
    return h;
}

// expander_init (expanders.h:47-60): C[dep], recurse, D[dep]
long long init_rec(GlibcRand& g, long long n, int dep, std::vector<HostGraph>& C, std::vector<HostGraph>& D)
{
    if (n <= kThreshold) return n;
    const long long R = c_targets(n);
    C.push_back(gen_graph(g, n, R, kCDegree));
    const long long L = init_rec(g, R, dep + 1, C, D);
    const long long RD = d_targets(n, L);
    HostGraph dg = gen_graph(g, L, RD, kDDegree);
    if ((long long)D.size() <= dep) D.resize(dep + 1);
    D[dep] = std::move(dg);
    return n + L + RD;
}

std::mutex g_mu;
std::map<std::pair<int, long long>, Encoder*> g_cache;

void state_to_bytes(const uint32_t st[8], unsigned char out[32])
{
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (unsigned char)(st[i] >> 24);
        out[4 * i + 1] = (unsigned char)(st[i] >> 16);
        out[4 * i + 2] = (unsigned char)(st[i] >> 8);
        out[4 * i + 3] = (unsigned char)st[i];
    }
}

// ---- kernels --------------------------------------------------------------

__device__ __forceinline__ ulonglong2 ldg16(const ulonglong2* p) { return __ldg(p); }


// out[c][r] = in[r][c] for in [n_r][n_c] (16-byte elements), 32 x 32 tiles,
// one tile per CTA in a 1-D grid
__global__ void __launch_bounds__(256) transpose_kernel(const ulonglong2* __restrict__ in,
                                                        ulonglong2* __restrict__ out,
                                                        long long n_r, long long n_c)
{
    __shared__ ulonglong2 tile[32][33];
    const long long tiles_c = (n_c + 31) / 32;
    const long long r0 = ((long long)blockIdx.x / tiles_c) * 32, c0 = ((long long)blockIdx.x % tiles_c) * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const long long r = r0 + ty + k, c = c0 + tx;
        if (r < n_r && c < n_c) tile[ty + k][tx] = ldg16(in + r * n_c + c);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const long long c = c0 + ty + k, r = r0 + tx;
        if (r < n_r && c < n_c) out[c * n_r + r] = tile[tx][ty + k];
    }
}

// splitmix64 (the reference's truepix::splitmix64) output number k + 1 from the
// state `seed`: the state after k + 1 increments is seed + (k + 1) * golden, so
// every private wire's mask is computed independently of the others.
__device__ __forceinline__ uint64_t zk_mask(uint64_t seed, long long k)
{
    uint64_t z = seed + (uint64_t)(k + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return canon61(z);   // z mod 2^61 - 1
}

// element f = copy * W + wire of the polynomial a PixelInput stands for
__device__ __forceinline__ uint64_t pixel_value(const PixelInput& px, long long f, int w_shift)
{
    const long long copy = f >> w_shift;
    const int wire = (int)(f & ((1LL << w_shift) - 1));
    if (copy >= px.copies) return 0;
    const bool priv = wire < px.cs;
    uint64_t v = 0;
    if (px.mask_mode != kMaskOnly) {
        if (priv)
            v = px.pix[copy * px.cs + wire];
        else if (wire == px.const_idx)
            v = px.const_val;
    }
    if (px.mask_mode != kMaskNone && priv) {
        const uint64_t m = zk_mask(px.mask_seed, copy * px.cs + wire);
        v = canon61(v + m);
    }
    return v;
}

// rows[r][c] = input element c * col_len + r of a frame (PixelInput layout)
// (and, when `bytes` is set, the same values as a row-major byte matrix
// bytes[r][c]: every value of an unmasked frame is < 256 when its constant is)
__global__ void __launch_bounds__(256) pixel_rows_kernel(PixelInput px, long long col_len, int w_shift,
                                                         ulonglong2* __restrict__ rows,
                                                         unsigned char* __restrict__ bytes)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= col_len * kColumns) return;
    const long long r = i >> 7, c = i & 127;
    const uint64_t v = pixel_value(px, c * col_len + r, w_shift);
    rows[i] = make_ulonglong2(0, v);
    if (bytes) bytes[i] = (unsigned char)v;
}

__global__ void __launch_bounds__(256) pixel_vector_kernel(PixelInput px, long long n, int w_shift,
                                                           uint64_t* __restrict__ out)
{
    const long long f = (long long)blockIdx.x * 256 + threadIdx.x;
    if (f < n) out[f] = pixel_value(px, f, w_shift);
}

// The depth-0 C multiplication of a frame, from its byte matrix: every source
// value v is < 2^8 with zero imaginary part, so w * v needs no field
// multiplication. With w = w1 * 2^32 + w0 (w0 < 2^32, w1 < 2^29), the sums
// S0 = sum w0 v < 2^(40 + 16) and S1 = sum w1 v stay exact in 64 bits for up to
// 2^16 in-edges (checked on the host), and S0 + S1 * 2^32 is reduced once per
// target. One warp per target row; lane l owns columns 4l .. 4l + 3, one 32-bit
// load (4 bytes) per edge.
__global__ void __launch_bounds__(256) gather_bytes_kernel(const unsigned char* __restrict__ bytes,
                                                           ulonglong2* __restrict__ rows, long long dst_row,
                                                           long long n_targets,
                                                           const unsigned* __restrict__ ptr,
                                                           const unsigned* __restrict__ esrc,
                                                           const ulonglong2* __restrict__ ew)
{
    const long long t = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (t >= n_targets) return;
    const int lane = threadIdx.x & 31;
    const unsigned e0 = ptr[t], e1 = ptr[t + 1];
    const uint32_t* src = reinterpret_cast<const uint32_t*>(bytes) + lane;
    // [column][re lo, re hi, im lo, im hi]
    u64 acc[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[k][q] = 0;
    for (unsigned eb = e0; eb < e1; eb += 32) {
        const int cnt = (int)min(32u, e1 - eb);
        unsigned my_s = 0;
        ulonglong2 my_w = make_ulonglong2(0, 0);
        if (lane < cnt) {
            my_s = esrc[eb + lane];
            my_w = ew[eb + lane];
        }
        for (int j = 0; j < cnt; ++j) {
            const unsigned sj = __shfl_sync(0xffffffffu, my_s, j);
            const uint32_t wr0 = __shfl_sync(0xffffffffu, (uint32_t)my_w.y, j);
            const uint32_t wr1 = __shfl_sync(0xffffffffu, (uint32_t)(my_w.y >> 32), j);
            const uint32_t wi0 = __shfl_sync(0xffffffffu, (uint32_t)my_w.x, j);
            const uint32_t wi1 = __shfl_sync(0xffffffffu, (uint32_t)(my_w.x >> 32), j);
            const uint32_t word = __ldg(src + (long long)sj * (kColumns / 4));
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t v = (word >> (8 * k)) & 0xFFu;
                acc[k][0] += (u64)wr0 * v;
                acc[k][1] += (u64)wr1 * v;
                acc[k][2] += (u64)wi0 * v;
                acc[k][3] += (u64)wi1 * v;
            }
        }
    }
    ulonglong2* dst = rows + (dst_row + t) * kColumns + 4 * lane;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const u64 re = acc[k][0] + ((acc[k][1] & 0x1FFFFFFFull) << 32) + (acc[k][1] >> 29);
        const u64 im = acc[k][2] + ((acc[k][3] & 0x1FFFFFFFull) << 32) + (acc[k][3] >> 29);
        dst[k] = make_ulonglong2(canon61(im), canon61(re));
    }
}

// One warp per target row t of a graph: rows[dst + t][c] = sum over in-edges
// (s, w) of w * rows[src + s][c]. Lane l owns columns l, l + 32, l + 64, l + 96
// (each edge reads one 2 KB row, 512 contiguous bytes per load instruction).
// Edge metadata is read 32 at a time, one edge per lane, and broadcast.
// The Fp2 products are accumulated as their three Karatsuba parts
// (sum xr wr, sum xi wi, sum (xr + xi)(wr + wi)), folded once per two edges,
// and combined into re = AC - BD, im = S - AC - BD once per target.
// CPL = columns per lane: 4 (one warp per target) for the large graphs, 1 (four
// warps per target, a quarter of the serial edge loop each) for the small ones,
// whose few targets would otherwise leave most SMs idle.
template <int CPL>
__global__ void __launch_bounds__(256) gather_kernel(ulonglong2* __restrict__ rows, long long src_row,
                                                     long long dst_row, long long n_targets,
                                                     const unsigned* __restrict__ ptr,
                                                     const unsigned* __restrict__ esrc,
                                                     const ulonglong2* __restrict__ ew)
{
    constexpr int kWarpsPerTarget = 4 / CPL;
    const long long gw = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    const long long t = gw / kWarpsPerTarget;
    const int sub = (int)(gw % kWarpsPerTarget);
    if (t >= n_targets) return;
    const int lane = threadIdx.x & 31;
    const unsigned e0 = ptr[t], e1 = ptr[t + 1];
    // column of slot k: lane + 32 (sub CPL + k)
    const ulonglong2* src = rows + src_row * kColumns + lane + 32 * sub * CPL;
    u64 ac[CPL], bd[CPL], sm[CPL];   // nearly canonical (< 2^61 + 8)
#pragma unroll
    for (int k = 0; k < CPL; ++k) ac[k] = bd[k] = sm[k] = 0;
    for (unsigned eb = e0; eb < e1; eb += 32) {
        const int cnt = (int)min(32u, e1 - eb);
        unsigned my_s = 0;
        ulonglong2 my_w = make_ulonglong2(0, 0);
        if (lane < cnt) {
            my_s = esrc[eb + lane];
            my_w = ew[eb + lane];
        }
        int j = 0;
        for (; j + 2 <= cnt; j += 2) {
            const unsigned s0 = __shfl_sync(0xffffffffu, my_s, j);
            const unsigned s1 = __shfl_sync(0xffffffffu, my_s, j + 1);
            const u64 w0r = __shfl_sync(0xffffffffu, my_w.y, j), w0i = __shfl_sync(0xffffffffu, my_w.x, j);
            const u64 w1r = __shfl_sync(0xffffffffu, my_w.y, j + 1), w1i = __shfl_sync(0xffffffffu, my_w.x, j + 1);
            const u64 w0s = w0r + w0i, w1s = w1r + w1i;   // < 2^62
            const ulonglong2* p0 = src + (long long)s0 * kColumns;
            const ulonglong2* p1 = src + (long long)s1 * kColumns;
            ulonglong2 v0[CPL], v1[CPL];
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                v0[k] = ldg16(p0 + 32 * k);
                v1[k] = ldg16(p1 + 32 * k);
            }
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                // three terms below 2^61 + 8 each: the sum stays below 2^63
                ac[k] = fold61(ac[k] + lmul(v0[k].y, w0r) + lmul(v1[k].y, w1r));
                bd[k] = fold61(bd[k] + lmul(v0[k].x, w0i) + lmul(v1[k].x, w1i));
                sm[k] = fold61(sm[k] + lmul(v0[k].y + v0[k].x, w0s) + lmul(v1[k].y + v1[k].x, w1s));
            }
        }
        if (j < cnt) {
            const unsigned s0 = __shfl_sync(0xffffffffu, my_s, j);
            const u64 w0r = __shfl_sync(0xffffffffu, my_w.y, j), w0i = __shfl_sync(0xffffffffu, my_w.x, j);
            const u64 w0s = w0r + w0i;
            const ulonglong2* p0 = src + (long long)s0 * kColumns;
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                const ulonglong2 v = ldg16(p0 + 32 * k);
                ac[k] = fold61(ac[k] + lmul(v.y, w0r));
                bd[k] = fold61(bd[k] + lmul(v.x, w0i));
                sm[k] = fold61(sm[k] + lmul(v.y + v.x, w0s));
            }
        }
    }
    ulonglong2* dst = rows + (dst_row + t) * kColumns + lane + 32 * sub * CPL;
#pragma unroll
    for (int k = 0; k < CPL; ++k) {
        const u64 re = fold61(ac[k] + (2 * P61 - bd[k]));
        const u64 im = fold61(sm[k] + (4 * P61 - ac[k] - bd[k]));
        dst[32 * k] = make_ulonglong2(canon61(im), canon61(re));
    }
}

constexpr int kLeafRows = 128;     // rows (threads) per CTA
constexpr int kLeafPairs = 4;      // column pairs staged per chunk

__device__ __forceinline__ void store_digest(unsigned char* tree, long long node, const uint32_t st[8])
{
    uint4 a, b;
    a.x = sha::bswap32(st[0]); a.y = sha::bswap32(st[1]); a.z = sha::bswap32(st[2]); a.w = sha::bswap32(st[3]);
    b.x = sha::bswap32(st[4]); b.y = sha::bswap32(st[5]); b.z = sha::bswap32(st[6]); b.w = sha::bswap32(st[7]);
    uint4* p = reinterpret_cast<uint4*>(tree + node * 32);
    p[0] = a;
    p[1] = b;
}

__device__ __forceinline__ void load_digest(const unsigned char* tree, long long node, uint32_t* w)
{
    const uint4* p = reinterpret_cast<const uint4*>(tree + node * 32);
    const uint4 a = p[0], b = p[1];
    w[0] = sha::bswap32(a.x); w[1] = sha::bswap32(a.y); w[2] = sha::bswap32(a.z); w[3] = sha::bswap32(a.w);
    w[4] = sha::bswap32(b.x); w[5] = sha::bswap32(b.y); w[6] = sha::bswap32(b.z); w[7] = sha::bswap32(b.w);
}

// Row leaves (linearPC.cpp:61-95,145-168): for row r < cw_len,
// h <- SHA256(h || rows[r][2j] || rows[r][2j+1]) for j = 0..63 from h = 0.
// One thread per row; the CTA stages 128 rows x 8 columns (padded to 9, so
// that 16-byte reads of consecutive rows fall in distinct banks) at a time.
// A launch covers the column pairs [pair0, pair1) (multiples of kLeafPairs): a
// chain split over several launches keeps its running state in the row's leaf
// slot (raw state words) between them, the last launch stores the digest bytes.
// Shorter launches free SMs sooner for other streams' kernels.
__global__ void __launch_bounds__(kLeafRows) leaf_kernel(const ulonglong2* __restrict__ rows, long long cw_len,
                                                         unsigned char* __restrict__ tree, long long leaf0,
                                                         uint32_t one, int pair0, int pair1)
{
    __shared__ ulonglong2 tile[kLeafRows][2 * kLeafPairs + 1];
    const long long r0 = (long long)blockIdx.x * kLeafRows;
    const int tid = threadIdx.x;
    const bool live = r0 + tid < cw_len;
    uint32_t* slot = reinterpret_cast<uint32_t*>(tree + (leaf0 + r0 + tid) * 32);
    uint32_t st[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) st[i] = (pair0 > 0 && live) ? slot[i] : 0;
    for (int pair = pair0; pair < pair1; pair += kLeafPairs) {
#pragma unroll
        for (int k = 0; k < 2 * kLeafPairs; ++k) {
            const int i = tid + k * kLeafRows;
            const int rr = i >> 3, cc = i & 7;
            const long long r = r0 + rr;
            tile[rr][cc] = r < cw_len ? ldg16(rows + r * kColumns + 2 * pair + cc) : make_ulonglong2(0, 0);
        }
        __syncthreads();
#pragma unroll 1
        for (int p = 0; p < kLeafPairs; ++p) {
            uint32_t w[16];
#pragma unroll
            for (int i = 0; i < 8; ++i) w[i] = st[i];
            const ulonglong2 x = tile[tid][2 * p], y = tile[tid][2 * p + 1];
            sha::fe_words(x.x, x.y, w + 8);
            sha::fe_words(y.x, y.y, w + 12);
            sha::hash64(w, st, sha::AddMad{one});
        }
        __syncthreads();
    }
    if (!live) return;
    if (pair1 == kColumns / 2) {
        store_digest(tree, leaf0 + r0 + tid, st);
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) slot[i] = st[i];
    }
}

// tree[leaf0 + i] for i in [from, to): `a` below `split`, `b` from there on
__global__ void fill_leaves_kernel(unsigned char* __restrict__ tree, long long leaf0, long long from,
                                   long long split, long long to, ulonglong2 a0, ulonglong2 a1,
                                   ulonglong2 b0, ulonglong2 b1)
{
    const long long i = from + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= to) return;
    ulonglong2* p = reinterpret_cast<ulonglong2*>(tree + (leaf0 + i) * 32);
    p[0] = i < split ? a0 : b0;
    p[1] = i < split ? a1 : b1;
}

// `levels` tree levels above the n_in nodes at heap positions [n_in, 2 n_in):
// CTA b reduces the 2^levels nodes from n_in + b * 2^levels to one node
// (merkle_tree.cpp:64-83: node k = SHA256(node 2k || node 2k + 1)).
__global__ void __launch_bounds__(256) tree_kernel(unsigned char* __restrict__ tree, long long n_in, int levels,
                                                   uint32_t one)
{
    __shared__ uint32_t s[256][9];
    const int t = threadIdx.x;
    long long base = n_in + ((long long)blockIdx.x << levels);   // first child of this level
    int cnt = 1 << (levels - 1);                                  // parents at this level
    uint32_t st[8];
    if (t < cnt) {
        uint32_t w[16];
        load_digest(tree, base + 2 * t, w);
        load_digest(tree, base + 2 * t + 1, w + 8);
        sha::hash64(w, st, sha::AddMad{one});
        store_digest(tree, (base >> 1) + t, st);
    }
    for (int lv = 1; lv < levels; ++lv) {
        if (t < cnt) {
#pragma unroll
            for (int i = 0; i < 8; ++i) s[t][i] = st[i];
        }
        __syncthreads();
        base >>= 1;
        cnt >>= 1;
        if (t < cnt) {
            uint32_t w[16];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                w[i] = s[2 * t][i];
                w[8 + i] = s[2 * t + 1][i];
            }
            sha::hash64(w, st, sha::AddMad{one});
            store_digest(tree, (base >> 1) + t, st);
        }
        __syncthreads();
    }
}

// Register-only throughput of the same SHA-256 code (the compute roof of the
// leaf kernels): every thread chains `iters` hashes of a 64-byte message made of
// its previous digest and a counter, no memory traffic.
__global__ void __launch_bounds__(kLeafRows) sha_peak_kernel(int iters, uint32_t one, uint32_t* out)
{
    uint32_t st[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) st[i] = threadIdx.x + 977u * blockIdx.x + i;
#pragma unroll 1
    for (int it = 0; it < iters; ++it) {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            w[i] = st[i];
            w[8 + i] = st[i] ^ (uint32_t)it;
        }
        sha::hash64(w, st, sha::AddMad{one});
    }
    atomicXor(out, st[0] ^ st[1] ^ st[2] ^ st[3] ^ st[4] ^ st[5] ^ st[6] ^ st[7]);
}

// The same gather for weights whose limbs are below 2^31 (Encoder::d_w32). For an
// element x = a + b i (canonical) and a weight c + d i, Karatsuba's three products
// a c, b d and s (c + d) with s = a + b reduced below p: each is a 61 x 32-bit
// product (< 2^93), accumulated exactly, by multiply-add with carry, into three
// 32-bit words (two 32 x 32 multiply-adds per product, no fold per product);
// every 8 edges each accumulator is folded mod 2^61 - 1 back below 2^61 + 8 (8
// products below 2^93 and the fold stay below 2^96). The result is
// (a c - b d) + (s (c + d) - a c - b d) i.
struct Acc3 {
    u32 w0, w1, w2;
};

__device__ __forceinline__ void mac32(Acc3& a, u64 x, u32 w)
{
    const u32 x0 = (u32)x, x1 = (u32)(x >> 32);
    asm("mad.lo.cc.u32 %0, %3, %5, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %5, %1;\n\t"
        "addc.u32 %2, %2, 0;\n\t"
        "mad.lo.cc.u32 %1, %4, %5, %1;\n\t"
        "madc.hi.u32 %2, %4, %5, %2;"
        : "+r"(a.w0), "+r"(a.w1), "+r"(a.w2)
        : "r"(x0), "r"(x1), "r"(w));
}

// the accumulator's value mod p, below 2^61 + 8 (2^64 == 8), stored back into it
__device__ __forceinline__ u64 settle(Acc3& a)
{
    const u64 lo = ((u64)a.w1 << 32) | a.w0;
    const u64 v = fold61(fold61(lo) + 8ull * a.w2);
    a.w0 = (u32)v;
    a.w1 = (u32)(v >> 32);
    a.w2 = 0;
    return v;
}

// one edge into the column's accumulators: element v {img, real}, weight c + d i, w = c + d
__device__ __forceinline__ void edge31(Acc3& A, Acc3& Bd, Acc3& S, ulonglong2 v, u32 c, u32 d, u32 w)
{
    u64 sum = v.y + v.x;
    sum = sum >= P61 ? sum - P61 : sum;
    mac32(A, v.y, c);
    mac32(Bd, v.x, d);
    mac32(S, sum, w);
}

template <int CPL>
__global__ void __launch_bounds__(256) gather31_kernel(ulonglong2* __restrict__ rows, long long src_row,
                                                       long long dst_row, long long n_targets,
                                                       const unsigned* __restrict__ ptr,
                                                       const unsigned* __restrict__ esrc,
                                                       const uint2* __restrict__ ew)
{
    constexpr int kWarpsPerTarget = 4 / CPL;
    const long long gw = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    const long long t = gw / kWarpsPerTarget;
    const int sub = (int)(gw % kWarpsPerTarget);
    if (t >= n_targets) return;
    const int lane = threadIdx.x & 31;
    const unsigned e0 = ptr[t], e1 = ptr[t + 1];
    const ulonglong2* src = rows + src_row * kColumns + lane + 32 * sub * CPL;
    Acc3 A[CPL], Bd[CPL], S[CPL];   // a c, b d, s (c + d)
#pragma unroll
    for (int k = 0; k < CPL; ++k) A[k] = Bd[k] = S[k] = Acc3{0, 0, 0};
    for (unsigned eb = e0; eb < e1; eb += 32) {
        const int cnt = (int)min(32u, e1 - eb);
        unsigned my_s = 0;
        uint2 my_w = make_uint2(0, 0);
        if (lane < cnt) {
            my_s = esrc[eb + lane];
            my_w = ew[eb + lane];
        }
        for (int h = 0; h < cnt; h += 8) {
            const int end = min(cnt, h + 8);
            int j = h;
            for (; j + 2 <= end; j += 2) {
                const unsigned s0 = __shfl_sync(0xffffffffu, my_s, j), s1 = __shfl_sync(0xffffffffu, my_s, j + 1);
                const u32 c0 = __shfl_sync(0xffffffffu, my_w.x, j), d0 = __shfl_sync(0xffffffffu, my_w.y, j);
                const u32 c1 = __shfl_sync(0xffffffffu, my_w.x, j + 1), d1 = __shfl_sync(0xffffffffu, my_w.y, j + 1);
                const ulonglong2* p0 = src + (long long)s0 * kColumns;
                const ulonglong2* p1 = src + (long long)s1 * kColumns;
                ulonglong2 v0[CPL], v1[CPL];
#pragma unroll
                for (int k = 0; k < CPL; ++k) {
                    v0[k] = ldg16(p0 + 32 * k);
                    v1[k] = ldg16(p1 + 32 * k);
                }
#pragma unroll
                for (int k = 0; k < CPL; ++k) {
                    edge31(A[k], Bd[k], S[k], v0[k], c0, d0, c0 + d0);
                    edge31(A[k], Bd[k], S[k], v1[k], c1, d1, c1 + d1);
                }
            }
            if (j < end) {
                const unsigned s0 = __shfl_sync(0xffffffffu, my_s, j);
                const u32 c0 = __shfl_sync(0xffffffffu, my_w.x, j), d0 = __shfl_sync(0xffffffffu, my_w.y, j);
                const ulonglong2* p0 = src + (long long)s0 * kColumns;
#pragma unroll
                for (int k = 0; k < CPL; ++k) edge31(A[k], Bd[k], S[k], ldg16(p0 + 32 * k), c0, d0, c0 + d0);
            }
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                settle(A[k]);
                settle(Bd[k]);
                settle(S[k]);
            }
        }
    }
    ulonglong2* dst = rows + (dst_row + t) * kColumns + lane + 32 * sub * CPL;
#pragma unroll
    for (int k = 0; k < CPL; ++k) {
        const u64 ac = settle(A[k]), bd = settle(Bd[k]), sw = settle(S[k]);
        dst[32 * k] = make_ulonglong2(canon61(fold61(sw + (4 * P61 - ac - bd))), canon61(fold61(ac + (2 * P61 - bd))));
    }
}

// graphs with fewer targets than this get four warps per target
constexpr long long kSmallGraph = 8192;

void launch_gather(ulonglong2* rows, long long src_row, long long dst_row, long long n_targets,
                   const unsigned* ptr, const unsigned* esrc, const ulonglong2* ew, const uint2* ew32,
                   cudaStream_t s)
{
    if (ew32) {
        const int cpl = n_targets < kSmallGraph ? 1 : g_gather_cpl.load();
        if (cpl == 1)
            gather31_kernel<1><<<(unsigned)((4 * n_targets + 7) / 8), 256, 0, s>>>(rows, src_row, dst_row,
                                                                                   n_targets, ptr, esrc, ew32);
        else if (cpl == 2)
            gather31_kernel<2><<<(unsigned)((2 * n_targets + 7) / 8), 256, 0, s>>>(rows, src_row, dst_row,
                                                                                   n_targets, ptr, esrc, ew32);
        else
            gather31_kernel<4><<<(unsigned)((n_targets + 7) / 8), 256, 0, s>>>(rows, src_row, dst_row, n_targets,
                                                                               ptr, esrc, ew32);
        return;
    }
    if (n_targets < kSmallGraph)
        gather_kernel<1><<<(unsigned)((4 * n_targets + 7) / 8), 256, 0, s>>>(rows, src_row, dst_row, n_targets,
                                                                             ptr, esrc, ew);
    else
        gather_kernel<4><<<(unsigned)((n_targets + 7) / 8), 256, 0, s>>>(rows, src_row, dst_row, n_targets, ptr,
                                                                         esrc, ew);
}

bool launch_ok(const char* what)
{
    ++g_launches;
    return !cuda_failed(cudaGetLastError(), what);
}

}  // namespace

long long codeword_len(long long col_len) { return cw_len_rec(col_len); }

long long tree_leaves(long long col_len)
{
    long long s = 1;
    while (s < 2 * col_len) s *= 2;
    return s;
}

void zero_row_leaf(unsigned char out[32])
{
    uint32_t st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < kColumns / 2; ++j) {
        uint32_t w[16];
        for (int i = 0; i < 8; ++i) w[i] = st[i];
        for (int i = 8; i < 16; ++i) w[i] = 0;
        sha::hash64(w, st);
    }
    state_to_bytes(st, out);
}

void zero_block_hash(unsigned char out[32])
{
    uint32_t w[16] = {0}, st[8];
    sha::hash64(w, st);
    state_to_bytes(st, out);
}

const Encoder* encoder(long long col_len)
{
    Ctx* c = ctx();
    if (!c) return nullptr;
    if (col_len < 1 || col_len > (1LL << 26)) {
        set_error(TP_ERR_ARG, "orion: column length %lld out of range [1, 2^26]", col_len);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    auto key = std::make_pair(c->device, col_len);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;

    GlibcRand g(1);
    std::vector<HostGraph> C, D;
    const long long cw = init_rec(g, col_len, 0, C, D);
    Encoder* e = new Encoder();
    e->device = c->device;
    e->col_len = col_len;
    e->cw_len = cw;
    std::vector<unsigned> ptr, src;
    std::vector<ulonglong2> w;
    long long off = 0, n = col_len;
    for (size_t k = 0; k < C.size(); ++k) {
        Level lv;
        lv.n = n;
        lv.R = C[k].R;
        lv.L = D[k].L;
        lv.RD = D[k].R;
        lv.off = off;
        lv.c_ptr = (long long)ptr.size();
        lv.c_edge = (long long)src.size();
        ptr.insert(ptr.end(), C[k].ptr.begin(), C[k].ptr.end());
        src.insert(src.end(), C[k].src.begin(), C[k].src.end());
        w.insert(w.end(), C[k].w.begin(), C[k].w.end());
        lv.d_ptr = (long long)ptr.size();
        lv.d_edge = (long long)src.size();
        ptr.insert(ptr.end(), D[k].ptr.begin(), D[k].ptr.end());
        src.insert(src.end(), D[k].src.begin(), D[k].src.end());
        w.insert(w.end(), D[k].w.begin(), D[k].w.end());
        e->levels.push_back(lv);
        off += n;
        n = lv.R;
    }
    if (!C.empty()) {
        unsigned mx = 0;
        for (size_t t = 0; t + 1 < C[0].ptr.size(); ++t) mx = std::max(mx, C[0].ptr[t + 1] - C[0].ptr[t]);
        e->max_c0_in_degree = mx;
    }
    e->n_ptr = (long long)ptr.size();
    e->n_edges = (long long)src.size();
    bool ok = true;
    if (e->n_ptr) ok = !cuda_failed(cudaMalloc(&e->d_ptr, sizeof(unsigned) * ptr.size()), "orion graph alloc");
    if (ok && e->n_edges) {
        ok = !cuda_failed(cudaMalloc(&e->d_src, sizeof(unsigned) * src.size()), "orion graph alloc") &&
             !cuda_failed(cudaMalloc(&e->d_w, sizeof(ulonglong2) * w.size()), "orion graph alloc");
    }
    if (ok && e->n_ptr)
        ok = !cuda_failed(cudaMemcpy(e->d_ptr, ptr.data(), sizeof(unsigned) * ptr.size(), cudaMemcpyHostToDevice),
                          "orion graph upload");
    if (ok && e->n_edges)
        ok = !cuda_failed(cudaMemcpy(e->d_src, src.data(), sizeof(unsigned) * src.size(), cudaMemcpyHostToDevice),
                          "orion graph upload") &&
             !cuda_failed(cudaMemcpy(e->d_w, w.data(), sizeof(ulonglong2) * w.size(), cudaMemcpyHostToDevice),
                          "orion graph upload");
    bool small = ok && e->n_edges > 0;
    for (size_t i = 0; small && i < w.size(); ++i) small = w[i].x < (1ull << 31) && w[i].y < (1ull << 31);
    if (small) {
        std::vector<uint2> w32(w.size());
        for (size_t i = 0; i < w.size(); ++i) w32[i] = make_uint2((unsigned)w[i].y, (unsigned)w[i].x);
        ok = !cuda_failed(cudaMalloc(&e->d_w32, sizeof(uint2) * w32.size()), "orion graph alloc") &&
             !cuda_failed(cudaMemcpy(e->d_w32, w32.data(), sizeof(uint2) * w32.size(), cudaMemcpyHostToDevice),
                          "orion graph upload");
    }
    if (!ok) {
        cudaFree(e->d_ptr);
        cudaFree(e->d_src);
        cudaFree(e->d_w);
        cudaFree(e->d_w32);
        delete e;
        return nullptr;
    }
    g_cache[key] = e;
    return e;
}

int last_launches() { return g_launches; }

bool set_gather_lanes(int columns_per_lane)
{
    if (columns_per_lane != 1 && columns_per_lane != 2 && columns_per_lane != 4) {
        set_error(TP_ERR_ARG, "orion: columns per lane %d not in {1, 2, 4}", columns_per_lane);
        return false;
    }
    g_gather_cpl.store(columns_per_lane);
    return true;
}

bool set_leaf_chunks(int n)
{
    if (n != 1 && n != 2 && n != 4 && n != 8 && n != 16) {
        set_error(TP_ERR_ARG, "leaf chunks %d: must be 1, 2, 4, 8 or 16", n);
        return false;
    }
    g_leaf_chunks.store(n);
    return true;
}
void add_launches(int n) { g_launches += n; }

bool sha_peak(int blocks, int iters, uint32_t* out, cudaStream_t s)
{
    sha_peak_kernel<<<blocks, kLeafRows, 0, s>>>(iters, 1u, out);
    return launch_ok("sha256 peak");
}

unsigned transpose_grid(long long n_r, long long n_c) { return (unsigned)(((n_r + 31) / 32) * ((n_c + 31) / 32)); }

bool rows_to_columns(const ulonglong2* rows, long long cw_len, ulonglong2* cols, cudaStream_t s)
{
    transpose_kernel<<<transpose_grid(cw_len, kColumns), 256, 0, s>>>(rows, cols, cw_len, kColumns);
    return launch_ok("orion rows_to_columns");
}

bool pixel_vector(const PixelInput& px, long long n, uint64_t* out, cudaStream_t s)
{
    int w_shift = 0;
    while ((1 << w_shift) < px.W) ++w_shift;
    pixel_vector_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(px, n, w_shift, out);
    return launch_ok("orion pixel vector");
}

bool commit(const Encoder& enc, const ulonglong2* src, const PixelInput* px, ulonglong2* rows,
            unsigned char* tree, cudaStream_t s)
{
    g_launches = 0;
    const long long col_len = enc.col_len, cw_len = enc.cw_len;
    const long long n_rows = 2 * col_len, size = tree_leaves(col_len);
    // node 0 of the heap is unused; the reference leaves it zero
    if (cuda_failed(cudaMemsetAsync(tree, 0, 32, s), "orion tree clear")) return false;
    // 1. the message: column-major input -> rows [0, col_len)
    unsigned char* bytes = nullptr;
    if (src) {
        timer_begin(s, kTagLoad);
        transpose_kernel<<<transpose_grid(kColumns, col_len), 256, 0, s>>>(src, rows, kColumns, col_len);
        timer_end(s);
        if (!launch_ok("orion load columns")) return false;
    } else {
        int w_shift = 0;
        while ((1 << w_shift) < px->W) ++w_shift;
        const long long n = col_len * kColumns;
        // byte path of the depth-0 C multiplication: values < 2^8, in-degree < 2^16
        if (px->mask_mode == kMaskNone && px->const_val < 256 && !enc.levels.empty() &&
            enc.max_c0_in_degree < (1u << 16)) {
            bytes = static_cast<unsigned char*>(dev_alloc((size_t)n, s));
            if (!bytes) return false;
        }
        timer_begin(s, kTagLoad);
        pixel_rows_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(*px, col_len, w_shift, rows, bytes);
        timer_end(s);
        if (!launch_ok("orion load pixels")) {
            if (bytes) dev_free(bytes, s);
            return false;
        }
    }
    // 2. C multiplications, outermost depth first
    for (const Level& lv : enc.levels) {
        if (lv.R == 0) continue;
        if (bytes && lv.off == 0) {
            timer_begin(s, kTagGatherBytes);
            gather_bytes_kernel<<<(unsigned)((lv.R + 7) / 8), 256, 0, s>>>(
                bytes, rows, lv.n, lv.R, enc.d_ptr + lv.c_ptr, enc.d_src + lv.c_edge, enc.d_w + lv.c_edge);
            timer_end(s);
            dev_free(bytes, s);
            bytes = nullptr;
            if (!launch_ok("orion C gather (bytes)")) return false;
            continue;
        }
        timer_begin(s, kTagGather);
        launch_gather(rows, lv.off, lv.off + lv.n, lv.R, enc.d_ptr + lv.c_ptr, enc.d_src + lv.c_edge,
                      enc.d_w + lv.c_edge, enc.d_w32 ? enc.d_w32 + lv.c_edge : nullptr, s);
        timer_end(s);
        if (!launch_ok("orion C gather")) return false;
    }
    if (bytes) dev_free(bytes, s);
    // 3. D multiplications, innermost depth first
    for (auto it = enc.levels.rbegin(); it != enc.levels.rend(); ++it) {
        const Level& lv = *it;
        if (lv.RD == 0) continue;
        const long long next = lv.off + lv.n;
        timer_begin(s, kTagGather);
        launch_gather(rows, next, next + lv.L, lv.RD, enc.d_ptr + lv.d_ptr, enc.d_src + lv.d_edge,
                      enc.d_w + lv.d_edge, enc.d_w32 ? enc.d_w32 + lv.d_edge : nullptr, s);
        timer_end(s);
        if (!launch_ok("orion D gather")) return false;
    }
    // 4. row leaves, constant leaves for the zero rows and the tree padding
    const int chunks = g_leaf_chunks.load();
    for (int k = 0; k < chunks; ++k) {
        timer_begin(s, kTagLeaf);
        leaf_kernel<<<(unsigned)((cw_len + kLeafRows - 1) / kLeafRows), kLeafRows, 0, s>>>(
            rows, cw_len, tree, size, 1u, k * (kColumns / 2) / chunks, (k + 1) * (kColumns / 2) / chunks);
        timer_end(s);
        if (!launch_ok("orion leaves")) return false;
    }
    if (size > cw_len) {
        unsigned char zr[32], zb[32];
        zero_row_leaf(zr);
        zero_block_hash(zb);
        ulonglong2 a[2], b[2];
        memcpy(a, zr, 32);
        memcpy(b, zb, 32);
        const long long n = size - cw_len;
        fill_leaves_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tree, size, cw_len, n_rows, size, a[0],
                                                                       a[1], b[0], b[1]);
        if (!launch_ok("orion fill leaves")) return false;
    }
    // 5. the tree
    return build_tree(tree, size, s);
}

bool leaf_digests(const ulonglong2* rows, long long count, unsigned char* digests, cudaStream_t s)
{
    if (count <= 0) return true;
    leaf_kernel<<<(unsigned)((count + kLeafRows - 1) / kLeafRows), kLeafRows, 0, s>>>(rows, count, digests, 0, 1u, 0,
                                                                                       kColumns / 2);
    return launch_ok("orion column leaves");
}

bool build_tree(unsigned char* tree, long long leaves, cudaStream_t s)
{
    // nine levels per launch
    long long n_in = leaves;
    while (n_in > 1) {
        int levels = 0;
        while (levels < 9 && (1LL << (levels + 1)) <= n_in) ++levels;
        const long long blocks = n_in >> levels;
        timer_begin(s, kTagTree);
        tree_kernel<<<(unsigned)blocks, 1 << (levels - 1), 0, s>>>(tree, n_in, levels, 1u);
        timer_end(s);
        if (!launch_ok("merkle tree")) return false;
        n_in >>= levels;
    }
    return true;
}

}  // namespace orion
}  // namespace tp
