// NNDescent's random start on the device — the draws of
// mlx_vis/_nndescent/nndescent.py:47-57 and 72-82, bit for bit.
//
// The reference takes them from NumPy's global legacy RandomState:
//   idx = randint(0, n - 1, (n, k), int32), shifted past the row's own index;
//   P   = float32(float32(randn(d, 100)) / sqrt(100))  when 100 < d;
//   P2  = float32(float32(randn(d, 300)) / sqrt(300))  when 300 < d.
// Those are MT19937 words (Matsumoto & Nishimura 1998) turned into bounded
// integers by masked rejection and into normals by Marsaglia's polar method on
// 53-bit doubles.  Every output depends on how many words the rejections before
// it consumed.
//
// Parallel path (with a workspace): the MT recurrence runs first and stores the
// raw state of every generation, enough words for the requested counts with a
// 10-sigma margin on the rejections (one CTA for short streams; segments of 65,536
// words on separate CTAs, started by jump-ahead, for long ones); the acceptance tests, ranks
// (block counts + scan) and output scatter then run over the whole grid, first
// for the integers, then for the normal pairs starting at the word where the
// integers stopped.  A final kernel rebuilds NumPy's state at the word where the
// draws stopped.  If the margin ever falls short (a status word in the
// workspace), a gated one-CTA walk, launched behind them and otherwise exiting at
// once, redoes all the draws from a copy of the incoming state.
// Sequential path (no workspace): the same one-CTA walk, generation by
// generation, testing and ranking each generation's 624 words in parallel.
//
// State buffer (uint32 words): key[624], pos, has_gauss, gauss (double, low word
// first), NumPy's get_state() layout.  No waits: every loop ends when the
// requested counts are produced or the generated words run out.
#include <math.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "scan.cuh"

namespace umapb {
namespace rstart {

constexpr int kN = 624, kM = 397, kHalf = kN - kM;  // 227
constexpr int kThreads = 640;
constexpr uint32_t kUpper = 0x80000000u, kLower = 0x7fffffffu, kMatrixA = 0x9908b0dfu;

__device__ __forceinline__ uint32_t mix(uint32_t a, uint32_t b) {
  const uint32_t y = (a & kUpper) | (b & kLower);
  return (y >> 1) ^ ((y & 1u) ? kMatrixA : 0u);
}

__device__ __forceinline__ uint32_t temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

// Next generation of o into w.  The published loop updates in place, so entry i
// reads the NEW entry i + M - N once i >= N - M, and the last entry reads the new
// entry 0: three phases of 227, 227 and 170 entries.
__device__ __forceinline__ void twist(const uint32_t* __restrict__ o, uint32_t* __restrict__ w) {
  for (int i = threadIdx.x; i < kHalf; i += blockDim.x) w[i] = o[i + kM] ^ mix(o[i], o[i + 1]);
  __syncthreads();
  for (int i = kHalf + threadIdx.x; i < 2 * kHalf; i += blockDim.x) w[i] = w[i - kHalf] ^ mix(o[i], o[i + 1]);
  __syncthreads();
  for (int i = 2 * kHalf + threadIdx.x; i < kN - 1; i += blockDim.x) w[i] = w[i - kHalf] ^ mix(o[i], o[i + 1]);
  if (threadIdx.x == 0) w[kN - 1] = w[kM - 1] ^ mix(o[kN - 1], w[0]);
  __syncthreads();
}

// Exclusive rank of this thread's flag among threads [0, t) and the block total.
__device__ __forceinline__ int block_rank(bool f, int* warp_sum, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, f);
  if (lane == 0) warp_sum[warp] = __popc(b);
  __syncthreads();
  int before = 0;
  total = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) {
    const int c = warp_sum[w];
    before += w < warp ? c : 0;
    total += c;
  }
  __syncthreads();
  return before + __popc(b & ((1u << lane) - 1u));
}

// 53-bit double in [0, 1) from two words: ((a >> 5) 2^26 + (b >> 6)) / 2^53 (exact)
__device__ __forceinline__ double unit53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// Where normal number g goes.  Projections (affine == 0): g < g1 into P, the rest
// into P2, as float32(float32(g) / s).  Affine (affine != 0): float32(loc + scale g)
// into P (RandomState.normal(loc, scale) cast to float32).
struct Out {
  int affine;
  int64_t g1;  // normals for P (d * 100, or 0)
  float* P;
  double s1;   // sqrt(100) as NumPy computes it; loc when affine
  float* P2;
  double s2;   // sqrt(300); scale when affine
};

__device__ __forceinline__ void emit(const Out& o, int64_t g, double v) {
  if (o.affine) {
    o.P[g] = __double2float_rn(__dadd_rn(o.s1, __dmul_rn(o.s2, v)));
    return;
  }
  const double x = (double)__double2float_rn(v);
  if (g < o.g1)
    o.P[g] = __double2float_rn(__ddiv_rn(x, o.s1));
  else
    o.P2[g - o.g1] = __double2float_rn(__ddiv_rn(x, o.s2));
}

// One CTA walks the stream from in_state and leaves the final state in state.
// With a gate, it runs only when *gate != 0 (the grid-wide path fell short).
__global__ void __launch_bounds__(kThreads) walk_kernel(const uint32_t* __restrict__ in_state,
                                                        uint32_t* __restrict__ state, const int32_t* __restrict__ gate,
                                                        int k, int64_t count, uint32_t rng, uint32_t mask,
                                                        int32_t* __restrict__ idx, int64_t G, Out out) {
  if (gate && *gate == 0) return;
  __shared__ uint32_t key[2][kN];
  __shared__ uint32_t words[kN + 4];
  __shared__ int warp_sum[kThreads / 32];
  __shared__ int s_pos, s_has;
  __shared__ double s_gauss;
  const int t = threadIdx.x;
  for (int i = t; i < kN; i += kThreads) key[0][i] = in_state[i];
  int pos = (int)in_state[kN];
  int has_gauss = (int)in_state[kN + 1];
  double gauss = __hiloint2double((int)in_state[kN + 3], (int)in_state[kN + 2]);
  int cur = 0;
  __syncthreads();

  // ---- bounded integers: accept (w & mask) <= rng ---------------------------
  if (rng == 0) {  // NumPy fills the constant and draws nothing
    for (int64_t q = t; q < count; q += kThreads) idx[q] = (q / k) == 0 ? 1 : 0;
  } else {
    int64_t produced = 0;
    while (produced < count) {
      if (pos >= kN) {
        twist(key[cur], key[cur ^ 1]);
        cur ^= 1;
        pos = 0;
      }
      const int p = pos + t;
      uint32_t v = 0;
      bool acc = false;
      if (p < kN) {
        v = temper(key[cur][p]) & mask;
        acc = v <= rng;
      }
      int total;
      const int r = block_rank(acc, warp_sum, total);
      const int64_t need = count - produced;
      if (acc && r < need) {
        const int64_t q = produced + r;
        idx[q] = (int32_t)((int64_t)v >= q / k ? v + 1u : v);
      }
      if (total >= need) {
        if (acc && r == need - 1) s_pos = p + 1;
        __syncthreads();
        pos = s_pos;
        produced = count;
      } else {
        produced += total;
        pos = kN;
      }
    }
  }

  // ---- normals (polar method), cached second value --------------------------
  if (G > 0) {
    int64_t made = 0;
    if (has_gauss) {
      if (t == 0) emit(out, 0, gauss);
      made = 1;
      has_gauss = 0;
      gauss = 0.0;
    }
    if (t == 0) {
      s_has = 0;
      s_gauss = 0.0;
    }
    int carry = 0;  // words of an incomplete attempt from the previous generation
    __syncthreads();
    while (made < G) {
      if (pos >= kN) {
        twist(key[cur], key[cur ^ 1]);
        cur ^= 1;
        pos = 0;
      }
      const int avail = kN - pos;
      if (t < avail) words[carry + t] = temper(key[cur][pos + t]);
      __syncthreads();
      const int len = carry + avail;
      const int A = len / 4;  // complete attempts (4 words each)
      bool acc = false;
      double x1 = 0.0, x2 = 0.0, r2 = 0.0;
      if (t < A) {
        x1 = 2.0 * unit53(words[4 * t], words[4 * t + 1]) - 1.0;
        x2 = 2.0 * unit53(words[4 * t + 2], words[4 * t + 3]) - 1.0;
        r2 = __dadd_rn(__dmul_rn(x1, x1), __dmul_rn(x2, x2));
        acc = r2 < 1.0 && r2 != 0.0;
      }
      int total;
      const int r = block_rank(acc, warp_sum, total);
      const int64_t need = G - made;
      const int64_t pairs = (need + 1) / 2;
      if (acc && r < pairs) {
        const double f = __dsqrt_rn(__ddiv_rn(-2.0 * log(r2), r2));
        const int64_t g = made + 2 * (int64_t)r;
        emit(out, g, __dmul_rn(f, x2));
        if (g + 1 < G) {
          emit(out, g + 1, __dmul_rn(f, x1));
        } else {
          s_has = 1;
          s_gauss = __dmul_rn(f, x1);
        }
      }
      if (total >= pairs) {
        if (acc && r == pairs - 1) s_pos = pos + (4 * t + 3 - carry) + 1;
        __syncthreads();
        pos = s_pos;
        has_gauss = s_has;
        gauss = s_gauss;
        made = G;
      } else {
        made += 2 * (int64_t)total;
        const int rem = len - 4 * A;
        if (t < rem) words[t] = words[4 * A + t];  // 4A >= 4 > rem unless A == 0 (then a no-op)
        carry = rem;
        pos = kN;
        __syncthreads();
      }
    }
  }

  // ---- final state ------------------------------------------------------------
  for (int i = t; i < kN; i += kThreads) state[i] = key[cur][i];
  if (t == 0) {
    state[kN] = (uint32_t)pos;
    state[kN + 1] = (uint32_t)has_gauss;
    state[kN + 2] = (uint32_t)__double2loint(gauss);
    state[kN + 3] = (uint32_t)__double2hiint(gauss);
  }
}


// ---- parallel path -------------------------------------------------------------
constexpr int kPar = 256;          // threads per block
constexpr int kIntPerBlock = 1024;  // stream words per block (4 per thread)
constexpr int kAttPerBlock = 512;   // normal attempts per block (2 per thread)

struct Scalars {
  int64_t tot_int, tot_att;  // accepted integers / attempts in the generated words
  int64_t int_stop;          // stream words the integers consumed
  int64_t end;               // stream words consumed after the normals
  double gauss_out;
  int32_t has_out;
  int32_t status;  // nonzero: the generated words fell short; the gated walk redoes the draws
};

// raw[n] = x_n of the MT sequence: x_0..x_623 is the incoming key (generation 0)
// and x_n = x_{n-227} ^ mix(x_{n-624}, x_{n-623}) for n >= 624, so raw[624 g + i] is
// word i of generation g.  mix is linear over GF(2) and x_{n-227}, x_{n-454} unfold
// by the same recurrence, so for n >= 1078
//   x_n = x_{n-681} ^ mix(x_{n-1078}, x_{n-1077}) ^ mix(x_{n-851}, x_{n-850})
//                   ^ mix(x_{n-624}, x_{n-623}),
// whose nearest operand is 623 words back: a block of 623 words depends only on
// earlier blocks, so one barrier covers 623 words (the plain recurrence allows 227).
// A run that starts at word n0 from the 624 words before it uses the plain
// recurrence for its first 454 words (two blocks of 227), then blocks of 623.  A
// block writes ring slots n mod 2048 that none of its reads touch (those lie
// 456..1700 slots away), so every block costs one barrier.
//
// One CTA generates about 3 words per ns, bound by its own instructions; longer
// streams are cut into segments of kSeg words that run on separate CTAs, each
// started from the 624 words before it, computed by jumping ahead:
//
// Jump-ahead.  Every bit position of x_n follows a linear recurrence over GF(2)
// whose characteristic polynomial is the generator's, phi, of degree 19937
// (Matsumoto & Nishimura 1998).  With r(x) = x^D mod phi(x) = sum_i r_i x^i,
//   x_{n+D} = XOR over {i : r_i = 1} of x_{n+i}     for every n >= 1
// (the low 31 bits of x_0 never enter the recurrence, hence n >= 1).  r depends on
// D only, not on the seed, so the host computes phi once (Berlekamp-Massey on one
// output bit of the generator) and the polynomials r for D = b kSeg (repeated
// multiplication by x^16384 reduced mod phi, whose terms below the leading one
// lie at least 623 exponents lower, so the reduction proceeds 64 bits at a time).
// On the device the 624 words that start segment b are XORs over a window of
// 19937 + 623 words that one CTA generated first.
constexpr int kStreamThreads = 640;
constexpr int kWide = 623;
constexpr int kRing = 2048;
constexpr int kDeg = 19937;                        // degree of phi
constexpr int kPolyWords = (kDeg + 63) / 64;       // 312 64-bit words per jump polynomial
constexpr int64_t kSeg = 65536;                    // words per segment
constexpr int kMaxJumps = 1024;                    // jump polynomials kept: segments 1..1024
constexpr int64_t kWinEnd = kN + (kDeg - 1) + kN;  // the window is x_624 .. x_21183
constexpr int kJumpParts = 32;                     // CTAs per segment start, one exponent range each
constexpr int kPartBits = 640;                     // exponents per CTA (10 polynomial words)
constexpr int kJumpThreads = 160;                  // a thread XORs words w, w + 160, w + 320, w + 480
static_assert(kJumpParts * kPartBits >= kDeg && kPartBits % 64 == 0, "jump ranges cover phi");

// row b - 1: x^(b kSeg) mod phi, bit i of word i / 64 = coefficient of x^i
__device__ uint64_t g_jump_poly[(size_t)kMaxJumps * kPolyWords];

// Words n0 .. end - 1; the ring holds x_{n0-624} .. x_{n0-1} at slots n mod 2048 and
// the caller has synchronised after filling it.
__device__ __forceinline__ void gen_words(uint32_t* ring, int64_t n0, int64_t end, uint32_t* __restrict__ raw) {
  constexpr uint32_t R = kRing - 1;
  const int t = threadIdx.x;
  const int64_t wide0 = n0 + 2 * kHalf;
  for (int64_t base = n0; base < wide0 && base < end; base += kHalf) {
    const int64_t n = base + t;
    if (t < kHalf && n < end) {
      const uint32_t m = (uint32_t)n;
      const uint32_t x = ring[(m - kHalf) & R] ^ mix(ring[(m - kN) & R], ring[(m - kN + 1) & R]);
      ring[m & R] = x;
      raw[n] = x;
    }
    __syncthreads();
  }
  for (int64_t base = wide0; base < end; base += kWide) {
    const int64_t n = base + t;
    if (t < kWide && n < end) {
      const uint32_t m = (uint32_t)n;
      const uint32_t x = ring[(m - 681) & R] ^ mix(ring[(m - 1078) & R], ring[(m - 1077) & R]) ^
                         mix(ring[(m - 851) & R], ring[(m - 850) & R]) ^ mix(ring[(m - 624) & R], ring[(m - 623) & R]);
      ring[m & R] = x;
      raw[n] = x;
    }
    __syncthreads();
  }
}

// raw[0 .. end): the incoming key, then x_624 .. x_{end-1}
__global__ void __launch_bounds__(kStreamThreads) stream_kernel(const uint32_t* __restrict__ state, int64_t end,
                                                                uint32_t* __restrict__ raw) {
  __shared__ uint32_t ring[kRing];
  for (int i = threadIdx.x; i < kN; i += kStreamThreads) {
    const uint32_t v = state[i];
    ring[i] = v;
    raw[i] = v;
  }
  __syncthreads();
  gen_words(ring, kN, end, raw);
}

// Partial start words of segment b = 1 + blockIdx.x / kJumpParts over the exponents
// [g kPartBits, (g + 1) kPartBits) of its polynomial, g = blockIdx.x % kJumpParts:
// part[(b - 1, g, w)] = XOR over those set exponents i of x_{624 + i + w}, w < 624.
__global__ void __launch_bounds__(kJumpThreads) jump_kernel(const uint32_t* __restrict__ raw,
                                                            uint32_t* __restrict__ part) {
  constexpr int kWinWords = kPartBits + 4 * kJumpThreads - 1;  // w up to 639 (words past 623 are unused)
  __shared__ uint32_t win[kWinWords];
  __shared__ uint16_t list[kPartBits];  // the set exponents, minus i0
  __shared__ int s_cnt;
  const int b1 = blockIdx.x / kJumpParts, g = blockIdx.x % kJumpParts;
  const int i0 = g * kPartBits;
  const int i1 = min(kDeg, i0 + kPartBits);
  const int t = threadIdx.x;
  const int have = i1 - i0 + kN - 1;  // x_{624 + i0} .. x_{624 + i1 + 622}, inside the window
  for (int u = t; u < kWinWords; u += kJumpThreads) win[u] = u < have ? raw[kN + i0 + u] : 0u;
  if (t < 32) {  // warp 0 lists the set exponents in increasing order (none at or past kDeg)
    const uint32_t* poly32 = reinterpret_cast<const uint32_t*>(g_jump_poly + (size_t)b1 * kPolyWords);
    int cnt = 0;
    for (int c = 0; c < kPartBits / 32; ++c) {
      const int q = i0 / 32 + c;
      const uint32_t word = q < 2 * kPolyWords ? poly32[q] : 0u;  // little-endian halves of the 64-bit words
      const bool set = (word >> t) & 1u;
      const unsigned bal = __ballot_sync(0xffffffffu, set);
      if (set) list[cnt + __popc(bal & ((1u << t) - 1u))] = (uint16_t)(c * 32 + t);
      cnt += __popc(bal);
    }
    if (t == 0) s_cnt = cnt;
  }
  __syncthreads();
  const int cnt = s_cnt;
  uint32_t acc[4] = {0u, 0u, 0u, 0u};
#pragma unroll 4
  for (int s = 0; s < cnt; ++s) {
    const int i = list[s];
#pragma unroll
    for (int u = 0; u < 4; ++u) acc[u] ^= win[i + t + u * kJumpThreads];  // i + w < kWinWords
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int w = t + u * kJumpThreads;
    if (w < kN) part[((size_t)b1 * kJumpParts + g) * kN + w] = acc[u];
  }
}

// Segment b = blockIdx.x generates x_n for n in [1248 + b kSeg, 1248 + (b + 1) kSeg)
// (the last one up to `total`) from x_{624 + b kSeg} .. x_{1247 + b kSeg}: for b = 0
// the window's words, else the XOR of the segment's kJumpParts partial words.
__global__ void __launch_bounds__(kStreamThreads) segment_kernel(const uint32_t* __restrict__ part, int64_t total,
                                                                 int nseg, uint32_t* __restrict__ raw) {
  __shared__ uint32_t ring[kRing];
  const int b = blockIdx.x, t = threadIdx.x;
  const int64_t s0 = kN + (int64_t)b * kSeg;
  const int64_t n0 = s0 + kN;
  const int64_t end = b == nseg - 1 ? total : min(total, n0 + kSeg);
  if (t < kN) {
    uint32_t v = 0u;
    if (b == 0) {
      v = raw[s0 + t];
    } else {
      const uint32_t* p = part + (size_t)(b - 1) * kJumpParts * kN + t;
#pragma unroll 8
      for (int g = 0; g < kJumpParts; ++g) v ^= p[(size_t)g * kN];
    }
    ring[(uint32_t)(s0 + t) & (kRing - 1)] = v;
  }
  __syncthreads();
  gen_words(ring, n0, end, raw);
}

// exclusive prefix of v over the block (kPar threads) and the block total
__device__ __forceinline__ int block_excl(int v, int* warp_tot, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  int before = 0;
  total = 0;
#pragma unroll
  for (int w = 0; w < kPar / 32; ++w) {
    const int c = warp_tot[w];
    before += w < warp ? c : 0;
    total += c;
  }
  __syncthreads();
  return before + x - v;
}

__device__ __forceinline__ uint32_t word_at(const uint32_t* raw, const uint32_t* state, int64_t w) {
  return temper(raw[(int64_t)state[kN] + w]);
}

__global__ void __launch_bounds__(kPar) int_count_kernel(const uint32_t* __restrict__ raw,
                                                         const uint32_t* __restrict__ state, int64_t Wi,
                                                         uint32_t rng, uint32_t mask, int32_t* __restrict__ counts) {
  __shared__ int warp_tot[kPar / 32];
  const int64_t w0 = (int64_t)blockIdx.x * kIntPerBlock + 4 * threadIdx.x;
  int c = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u)
    if (w0 + u < Wi) c += (word_at(raw, state, w0 + u) & mask) <= rng ? 1 : 0;
  int total;
  block_excl(c, warp_tot, total);
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kPar) int_scatter_kernel(const uint32_t* __restrict__ raw,
                                                           const uint32_t* __restrict__ state, int64_t Wi,
                                                           uint32_t rng, uint32_t mask,
                                                           const int32_t* __restrict__ offsets, int64_t count, int k,
                                                           int32_t* __restrict__ idx, Scalars* sc) {
  __shared__ int warp_tot[kPar / 32];
  const int64_t w0 = (int64_t)blockIdx.x * kIntPerBlock + 4 * threadIdx.x;
  uint32_t v[4];
  bool acc[4];
  int c = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    v[u] = w0 + u < Wi ? word_at(raw, state, w0 + u) & mask : 0xffffffffu;
    acc[u] = w0 + u < Wi && v[u] <= rng;
    c += acc[u] ? 1 : 0;
  }
  int total;
  int64_t r = offsets[blockIdx.x] + block_excl(c, warp_tot, total);
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    if (!acc[u]) continue;
    if (r < count) idx[r] = (int32_t)((int64_t)v[u] >= r / k ? v[u] + 1u : v[u]);
    if (r == count - 1) sc->int_stop = w0 + u + 1;
    ++r;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && sc->tot_int < count) atomicOr(&sc->status, 1);
}

// attempt a of the normals uses stream words int_stop + 4a .. + 3
__device__ __forceinline__ bool attempt(const uint32_t* raw, const uint32_t* state, int64_t w, double& x1,
                                        double& x2, double& r2) {
  x1 = 2.0 * unit53(word_at(raw, state, w), word_at(raw, state, w + 1)) - 1.0;
  x2 = 2.0 * unit53(word_at(raw, state, w + 2), word_at(raw, state, w + 3)) - 1.0;
  r2 = __dadd_rn(__dmul_rn(x1, x1), __dmul_rn(x2, x2));
  return r2 < 1.0 && r2 != 0.0;
}

__global__ void __launch_bounds__(kPar) att_count_kernel(const uint32_t* __restrict__ raw,
                                                         const uint32_t* __restrict__ state, const Scalars* sc,
                                                         int64_t Aw, int32_t* __restrict__ counts) {
  __shared__ int warp_tot[kPar / 32];
  const int64_t a0 = (int64_t)blockIdx.x * kAttPerBlock + 2 * threadIdx.x;
  const int64_t s = sc->int_stop;
  int c = 0;
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    double x1, x2, r2;
    if (a0 + u < Aw) c += attempt(raw, state, s + 4 * (a0 + u), x1, x2, r2) ? 1 : 0;
  }
  int total;
  block_excl(c, warp_tot, total);
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kPar) att_scatter_kernel(const uint32_t* __restrict__ raw,
                                                           const uint32_t* __restrict__ state, Scalars* sc, int64_t Aw,
                                                           const int32_t* __restrict__ offsets, int64_t G, Out out) {
  __shared__ int warp_tot[kPar / 32];
  const int64_t a0 = (int64_t)blockIdx.x * kAttPerBlock + 2 * threadIdx.x;
  const int64_t s = sc->int_stop;
  const int made0 = state[kN + 1] ? 1 : 0;  // a cached normal is used first
  const int64_t pairs = (G - made0 + 1) / 2;
  double x1[2], x2[2], r2[2];
  bool acc[2];
  int c = 0;
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    acc[u] = a0 + u < Aw && attempt(raw, state, s + 4 * (a0 + u), x1[u], x2[u], r2[u]);
    c += acc[u] ? 1 : 0;
  }
  int total;
  int64_t r = offsets[blockIdx.x] + block_excl(c, warp_tot, total);
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    if (!acc[u]) continue;
    if (r < pairs) {
      const double f = __dsqrt_rn(__ddiv_rn(-2.0 * log(r2[u]), r2[u]));
      const int64_t g = made0 + 2 * r;
      emit(out, g, __dmul_rn(f, x2[u]));
      if (g + 1 < G) {
        emit(out, g + 1, __dmul_rn(f, x1[u]));
      } else {
        sc->has_out = 1;
        sc->gauss_out = __dmul_rn(f, x1[u]);
      }
    }
    if (r == pairs - 1) sc->end = s + 4 * (a0 + u) + 4;
    ++r;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (made0) emit(out, 0, __hiloint2double((int)state[kN + 3], (int)state[kN + 2]));
    if (sc->tot_att < pairs) atomicOr(&sc->status, 2);
  }
}

// NumPy's state after `consumed` stream words (and the normals' cache)
__global__ void __launch_bounds__(kPar) final_state_kernel(const uint32_t* __restrict__ raw,
                                                           uint32_t* __restrict__ state, const Scalars* sc,
                                                           int64_t G) {
  const int64_t pos0 = state[kN];
  const int made0 = state[kN + 1] ? 1 : 0;
  const int64_t pairs = G > 0 ? (G - made0 + 1) / 2 : 0;
  const int64_t consumed = pairs > 0 ? sc->end : sc->int_stop;
  __syncthreads();  // every thread has read the incoming state
  if (consumed > 0) {
    const int64_t e = pos0 + consumed;  // raw index after the last consumed word
    const int64_t gen = (e - 1) / kN;
    for (int i = threadIdx.x; i < kN; i += kPar) state[i] = raw[gen * kN + i];
    if (threadIdx.x == 0) state[kN] = (uint32_t)(e - gen * kN);
  }
  if (threadIdx.x == 0 && G > 0) {
    const int has = pairs > 0 ? sc->has_out : 0;
    const double gs = pairs > 0 && has ? sc->gauss_out : 0.0;
    state[kN + 1] = (uint32_t)has;
    state[kN + 2] = (uint32_t)__double2loint(gs);
    state[kN + 3] = (uint32_t)__double2hiint(gs);
  }
}

__global__ void const_ints_kernel(int64_t count, int k, int32_t* __restrict__ idx) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
    idx[q] = (q / k) == 0 ? 1 : 0;
}

// ---- jump polynomials (host) ---------------------------------------------------
namespace jumps {
constexpr int kShift = 16384;                   // x^kSeg = (x^kShift)^4
constexpr int kBuf = (kDeg + kShift) / 64 + 2;  // words of a product before its reduction
constexpr int kMaxDev = 64;

inline uint32_t mix_h(uint32_t a, uint32_t b) {
  const uint32_t y = (a & kUpper) | (b & kLower);
  return (y >> 1) ^ ((y & 1u) ? kMatrixA : 0u);
}

// bits [pos, pos + 64) of a bit array, zero past its end
inline uint64_t get64(const std::vector<uint64_t>& a, int64_t pos) {
  const size_t q = (size_t)(pos >> 6);
  const int s = (int)(pos & 63);
  const uint64_t lo = q < a.size() ? a[q] : 0ull;
  const uint64_t hi = q + 1 < a.size() ? a[q + 1] : 0ull;
  return s ? (lo >> s) | (hi << (64 - s)) : lo;
}

// C ^= B x^m (terms past C's end are zero by the callers' degree bounds)
inline void xor_shift(std::vector<uint64_t>& C, const std::vector<uint64_t>& B, int m) {
  const int a = m >> 6, s = m & 63;
  for (int q = (int)C.size() - 1; q >= a; --q) {
    uint64_t v = B[q - a] << s;
    if (s && q - a - 1 >= 0) v |= B[q - a - 1] >> (64 - s);
    C[q] ^= v;
  }
}

// phi by Berlekamp-Massey (Massey 1969) on the top bit of 2 kDeg + 64 raw words of
// the recurrence from an arbitrary state.  exps: phi's exponents below kDeg, in
// decreasing order.  Fails unless the linear complexity is kDeg, phi(0) = 1 and the
// highest exponent below kDeg is at least 64 lower (the reduction's step).
bool char_poly(std::vector<int>& exps) {
  constexpr int N = 2 * kDeg + 64;
  constexpr int skip = 4 * kN;
  std::vector<uint32_t> x((size_t)kN + skip + N);
  uint32_t v = 2463534242u;  // xorshift32 (Marsaglia 2003) fills the first generation
  for (int i = 0; i < kN; ++i) {
    v ^= v << 13;
    v ^= v >> 17;
    v ^= v << 5;
    x[i] = v;
  }
  for (size_t n = kN; n < x.size(); ++n) x[n] = x[n - kHalf] ^ mix_h(x[n - kN], x[n - kN + 1]);
  const int words = N / 64 + 4;
  std::vector<uint64_t> rv(words, 0ull);  // bit j = s_{N-1-j}, s_j = top bit of x_{624 + skip + j}
  for (int j = 0; j < N; ++j)
    if (x[(size_t)kN + skip + j] >> 31) {
      const int p = N - 1 - j;
      rv[p >> 6] |= 1ull << (p & 63);
    }
  std::vector<uint64_t> C(words, 0ull), B(words, 0ull), T;
  C[0] = B[0] = 1ull;
  int L = 0, m = 1;
  for (int n = 0; n < N; ++n) {
    const int64_t base = (int64_t)N - 1 - n;  // rv bit of s_n; s_{n-i} is bit base + i
    uint64_t d = 0ull;
    for (int q = 0; q <= L / 64; ++q) d ^= C[q] & get64(rv, base + 64 * q);
    if ((__builtin_popcountll(d) & 1) == 0) {
      ++m;
    } else if (2 * L <= n) {
      T = C;
      xor_shift(C, B, m);
      L = n + 1 - L;
      B.swap(T);
      m = 1;
    } else {
      xor_shift(C, B, m);
      ++m;
    }
  }
  if (L != kDeg || !((C[L >> 6] >> (L & 63)) & 1ull)) return false;
  exps.clear();
  for (int i = 1; i <= L; ++i)  // phi(x) = x^L C(1/x): coefficient of x^(L - i) is c_i
    if ((C[i >> 6] >> (i & 63)) & 1ull) exps.push_back(L - i);
  return !exps.empty() && exps.back() == 0 && exps.front() <= kDeg - 64;
}

inline void xor_at(uint64_t* w, int pos, uint64_t v) {
  if (pos < 0) {  // only the partial top word: its bits below -pos are zero
    v >>= -pos;
    pos = 0;
  }
  const int q = pos >> 6, s = pos & 63;
  w[q] ^= v << s;
  if (s) w[q + 1] ^= v >> (64 - s);
}

// w <- w x^s mod phi for w of degree < kDeg (kBuf words), s <= kShift.  The top
// 64-bit word above x^kDeg folds down through x^kDeg = sum of x^e over exps: every
// image lies at least 623 - 63 bits below the word, so one pass from the top works.
void mulx_mod(uint64_t* w, int s, const std::vector<int>& exps) {
  const int a = s >> 6, b = s & 63;
  for (int q = kBuf - 1; q >= 0; --q) {
    uint64_t v = q - a >= 0 ? w[q - a] << b : 0ull;
    if (b && q - a - 1 >= 0) v |= w[q - a - 1] >> (64 - b);
    w[q] = v;
  }
  for (int q = kBuf - 1; q >= kDeg / 64; --q) {
    uint64_t v = w[q];
    if (q == kDeg / 64) v &= ~0ull << (kDeg & 63);
    if (!v) continue;
    w[q] ^= v;
    for (int e : exps) xor_at(w, 64 * q - kDeg + e, v);
  }
}

struct Table {
  std::mutex mu;
  bool tried = false, ok = false;
  std::vector<int> exps;
  std::vector<uint64_t> cur;    // x^(count kSeg) mod phi, kBuf words
  std::vector<uint64_t> polys;  // count rows of kPolyWords: x^(b kSeg) mod phi, b = 1..count
  int count = 0;
  int uploaded[kMaxDev] = {};   // rows in each device's g_jump_poly
};

Table& table() {
  static Table t;
  return t;
}

// the first `need` rows on the host; the caller holds the lock
bool extend(Table& T, int need) {
  if (!T.tried) {
    T.tried = true;
    T.ok = char_poly(T.exps);
    if (T.ok) {
      T.cur.assign(kBuf, 0ull);
      T.cur[0] = 1ull;
    }
  }
  if (!T.ok) return false;
  while (T.count < need) {
    for (int s = 0; s < kSeg / kShift; ++s) mulx_mod(T.cur.data(), kShift, T.exps);
    T.polys.insert(T.polys.end(), T.cur.begin(), T.cur.begin() + kPolyWords);
    ++T.count;
  }
  return true;
}
}  // namespace jumps

// Rows 1..need of g_jump_poly on the current device.  A first upload (one per device
// and table size) is synchronised on `stream`, so it is skipped, and the one-CTA
// stream used instead, while the stream is being captured.
static bool jump_table_ready(int need, cudaStream_t stream) {
  int dev = 0;
  if (need < 1 || need > kMaxJumps || cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= jumps::kMaxDev)
    return false;
  jumps::Table& T = jumps::table();
  std::lock_guard<std::mutex> lock(T.mu);
  if (!jumps::extend(T, need)) return false;
  if (T.uploaded[dev] >= need) return true;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return false;
  }
  const size_t off = (size_t)T.uploaded[dev] * kPolyWords;
  const size_t words = (size_t)need * kPolyWords - off;
  if (cudaMemcpyToSymbolAsync(g_jump_poly, T.polys.data() + off, words * sizeof(uint64_t), off * sizeof(uint64_t),
                              cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  T.uploaded[dev] = need;
  return true;
}

// Segments of x_1248 .. x_{total-1}; 1 means one CTA generates the whole stream.
static int segments(int64_t total) {
  if (total < kWinEnd + kSeg) return 1;
  const int64_t s = ceil_div(total - 2 * kN, kSeg);
  return (int)(s < kMaxJumps + 1 ? s : kMaxJumps + 1);  // the last segment runs to the end
}

struct Plan {
  int64_t Wi, Aw, n_gen, nbI, nbA;
  int nseg;
  size_t bytes;
  Scalars* sc;
  uint32_t* backup;  // the incoming state, for the gated walk
  uint32_t* raw;
  uint32_t* part;    // (nseg - 1, kJumpParts, 624) partial start words of the segments
  int32_t* cnt_i;
  int32_t* cnt_a;
  int64_t* scan_ws;  // scan_exclusive's block totals
};

// Words for `count` integers accepted with probability p = (rng + 1) / (mask + 1)
// and for the normal pairs (probability pi / 4), each with a 10-sigma margin.
static Plan plan(void* ws, int64_t count, uint32_t rng, uint32_t mask, int64_t G) {
  Plan p{};
  if (count > 0 && rng > 0) {
    const double q = ((double)rng + 1.0) / ((double)mask + 1.0);
    p.Wi = (int64_t)ceil(count / q + 10.0 * sqrt(count * (1.0 - q)) / q) + 64;
  }
  if (G > 0) {
    const double q = 0.78539816339744830962;
    const double pairs = (double)((G + 1) / 2);
    p.Aw = (int64_t)ceil(pairs / q + 10.0 * sqrt(pairs * (1.0 - q)) / q) + 64;
  }
  p.n_gen = (kN + p.Wi + 4 * p.Aw + kN - 1) / kN + 1;
  p.nbI = (p.Wi + kIntPerBlock - 1) / kIntPerBlock;
  p.nbA = (p.Aw + kAttPerBlock - 1) / kAttPerBlock;
  Carver c(ws);
  p.sc = c.take<Scalars>(1);
  p.backup = c.take<uint32_t>(kN + 4);
  p.raw = c.take<uint32_t>((size_t)(p.n_gen + 1) * kN);
  p.nseg = segments((p.n_gen + 1) * kN);
  p.part = c.take<uint32_t>((size_t)(p.nseg - 1) * kJumpParts * kN);
  p.cnt_i = c.take<int32_t>((size_t)p.nbI + 1);
  p.cnt_a = c.take<int32_t>((size_t)p.nbA + 1);
  p.scan_ws = c.take<int64_t>(kScanMaxBlocks);
  p.bytes = c.bytes();
  return p;
}

static int run_parallel(const Plan& p, uint32_t* state, int64_t count, int k, uint32_t rng, uint32_t mask,
                        int32_t* idx, int64_t G, const Out& out, cudaStream_t stream) {
  UMAPB_CUDA_TRY(cudaMemsetAsync(p.sc, 0, sizeof(Scalars), stream), "random draws: reset");
  UMAPB_CUDA_TRY(cudaMemcpyAsync(p.backup, state, (kN + 4) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream),
                 "random draws: state copy");
  int launches = 3;
  const int64_t total = (p.n_gen + 1) * kN;
  if (p.nseg > 1 && jump_table_ready(p.nseg - 1, stream)) {
    stream_kernel<<<1, kStreamThreads, 0, stream>>>(state, kWinEnd, p.raw);
    jump_kernel<<<(unsigned)((p.nseg - 1) * kJumpParts), kJumpThreads, 0, stream>>>(p.raw, p.part);
    segment_kernel<<<(unsigned)p.nseg, kStreamThreads, 0, stream>>>(p.part, total, p.nseg, p.raw);
    launches += 2;
  } else {
    stream_kernel<<<1, kStreamThreads, 0, stream>>>(state, total, p.raw);
  }
  if (count > 0 && rng == 0) {
    const int64_t want = (count + 255) / 256;
    const_ints_kernel<<<(unsigned)(want < 4096 ? want : 4096), 256, 0, stream>>>(count, k, idx);
    ++launches;
  } else if (count > 0) {
    int_count_kernel<<<(unsigned)p.nbI, kPar, 0, stream>>>(p.raw, state, p.Wi, rng, mask, p.cnt_i);
    scan_exclusive(p.cnt_i, p.nbI, &p.sc->tot_int, p.scan_ws, stream);
    int_scatter_kernel<<<(unsigned)p.nbI, kPar, 0, stream>>>(p.raw, state, p.Wi, rng, mask, p.cnt_i, count, k, idx,
                                                             p.sc);
    launches += 3;
  }
  if (G > 0) {
    att_count_kernel<<<(unsigned)p.nbA, kPar, 0, stream>>>(p.raw, state, p.sc, p.Aw, p.cnt_a);
    scan_exclusive(p.cnt_a, p.nbA, &p.sc->tot_att, p.scan_ws, stream);
    att_scatter_kernel<<<(unsigned)p.nbA, kPar, 0, stream>>>(p.raw, state, p.sc, p.Aw, p.cnt_a, G, out);
    launches += 3;
  }
  final_state_kernel<<<1, kPar, 0, stream>>>(p.raw, state, p.sc, G);
  // exits at once unless a margin fell short; then redoes every draw from the backup
  walk_kernel<<<1, kThreads, 0, stream>>>(p.backup, state, &p.sc->status, k, count, rng, mask, idx, G, out);
  UMAPB_LAUNCH_CHECK("random draws kernels");
  count_launches(launches);
  return UMAPB_OK;
}
}  // namespace rstart
}  // namespace umapb

using namespace umapb;

static void mask_of(int64_t n, uint32_t* rng, uint32_t* mask) {
  *rng = (uint32_t)(n - 2);  // randint(0, n - 1): values 0 .. n - 2
  uint32_t m = *rng;
  for (int s = 1; s <= 16; s <<= 1) m |= m >> s;
  *mask = m;
}

extern "C" int umapb_nnd_random_start_workspace(int64_t n, int32_t k, int32_t d, int32_t pd1, int32_t pd2,
                                                size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes && n >= 2 && n - 1 <= 0x7fffffff && k >= 1 && d >= 1 && pd1 >= 0 && pd2 >= 0,
                "nnd_random_start_workspace: bad arguments");
  uint32_t rng, mask;
  mask_of(n, &rng, &mask);
  *bytes = rstart::plan(nullptr, n * (int64_t)k, rng, mask, (int64_t)d * (pd1 + pd2)).bytes;
  return UMAPB_OK;
}

extern "C" int umapb_nnd_random_start(uint32_t* state, int64_t n, int32_t k, int32_t d, int32_t* idx, float* P,
                                      int32_t pd1, float* P2, int32_t pd2, void* workspace, size_t workspace_bytes,
                                      umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(state && idx, "nnd_random_start: null state or idx");
  UMAPB_REQUIRE(n >= 2 && n - 1 <= 0x7fffffff && k >= 1 && d >= 1, "nnd_random_start: need n >= 2, k >= 1, d >= 1");
  UMAPB_REQUIRE(pd1 >= 0 && pd2 >= 0 && (pd1 == 0 || P) && (pd2 == 0 || P2),
                "nnd_random_start: projection sizes must be >= 0 with their outputs given");
  uint32_t rng, mask;
  mask_of(n, &rng, &mask);
  rstart::Out out;
  out.affine = 0;
  out.g1 = (int64_t)d * pd1;
  out.P = P;
  out.s1 = sqrt((double)(pd1 > 0 ? pd1 : 1));
  out.P2 = P2;
  out.s2 = sqrt((double)(pd2 > 0 ? pd2 : 1));
  const int64_t G = out.g1 + (int64_t)d * pd2;
  const int64_t count = n * (int64_t)k;
  if (workspace) {
    const rstart::Plan need = rstart::plan(nullptr, count, rng, mask, G);
    if (workspace_bytes < need.bytes)
      return set_error(UMAPB_ERR_WORKSPACE, "nnd_random_start: workspace of %zu bytes, need %zu", workspace_bytes,
                       need.bytes);
    return rstart::run_parallel(rstart::plan(workspace, count, rng, mask, G), state, count, k, rng, mask, idx, G,
                                out, stream);
  }
  rstart::walk_kernel<<<1, rstart::kThreads, 0, stream>>>(state, state, nullptr, k, count, rng, mask, idx, G, out);
  UMAPB_LAUNCH_CHECK("nnd_random_start kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_legacy_normal_workspace(int64_t count, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes && count >= 0, "legacy_normal_workspace: bad arguments");
  *bytes = rstart::plan(nullptr, 0, 1u, 1u, count).bytes;
  return UMAPB_OK;
}

extern "C" int umapb_legacy_normal(uint32_t* state, int64_t count, double loc, double scale, float* out,
                                   void* workspace, size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(state && (out || count == 0) && count >= 0, "legacy_normal: bad arguments");
  if (count == 0) return UMAPB_OK;
  rstart::Out o;
  o.affine = 1;
  o.g1 = count;
  o.P = out;
  o.s1 = loc;
  o.P2 = nullptr;
  o.s2 = scale;
  if (workspace) {
    const rstart::Plan need = rstart::plan(nullptr, 0, 1u, 1u, count);
    if (workspace_bytes < need.bytes)
      return set_error(UMAPB_ERR_WORKSPACE, "legacy_normal: workspace of %zu bytes, need %zu", workspace_bytes,
                       need.bytes);
    return rstart::run_parallel(rstart::plan(workspace, 0, 1u, 1u, count), state, 0, 1, 1u, 1u, nullptr, count, o,
                                stream);
  }
  // no bounded integers (count 0): the walk goes straight to the normals
  rstart::walk_kernel<<<1, rstart::kThreads, 0, stream>>>(state, state, nullptr, 1, 0, 1u, 1u, nullptr, count, o);
  UMAPB_LAUNCH_CHECK("legacy_normal kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_mt_jump_poly(int32_t b, uint64_t* out, int64_t* words_ahead) {
  clear_error();
  UMAPB_REQUIRE(out && b >= 1 && b <= rstart::kMaxJumps, "mt_jump_poly: need 1 <= b <= %d and an output",
                rstart::kMaxJumps);
  rstart::jumps::Table& T = rstart::jumps::table();
  std::lock_guard<std::mutex> lock(T.mu);
  if (!rstart::jumps::extend(T, b))
    return set_error(UMAPB_ERR_UNSUPPORTED, "mt_jump_poly: the characteristic polynomial was not found");
  for (int q = 0; q < rstart::kPolyWords; ++q) out[q] = T.polys[(size_t)(b - 1) * rstart::kPolyWords + q];
  if (words_ahead) *words_ahead = (int64_t)b * rstart::kSeg;
  return UMAPB_OK;
}
