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
// it consumed, so the stream is walked by one CTA: 640 threads hold one state
// word each, a generation (twist) takes three dependent phases, and each
// generation's 624 words are tested, ranked with a block scan and scattered to
// their output slots in parallel.  The state enters and leaves in NumPy's
// get_state() layout, so the host hands the stream back to NumPy afterwards.
//
// State buffer (uint32 words): key[624], pos, has_gauss, gauss (double, low word
// first).  No waits: the loops end when the requested counts are produced.
#include <math.h>

#include "common.cuh"

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
  const int t = threadIdx.x;
  if (t < kHalf) w[t] = o[t + kM] ^ mix(o[t], o[t + 1]);
  __syncthreads();
  if (t >= kHalf && t < 2 * kHalf) w[t] = w[t - kHalf] ^ mix(o[t], o[t + 1]);
  __syncthreads();
  if (t >= 2 * kHalf && t < kN - 1) w[t] = w[t - kHalf] ^ mix(o[t], o[t + 1]);
  if (t == kN - 1) w[t] = w[kM - 1] ^ mix(o[kN - 1], w[0]);
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

__global__ void __launch_bounds__(kThreads) random_start_kernel(uint32_t* __restrict__ state, int k, int64_t count,
                                                                uint32_t rng, uint32_t mask,
                                                                int32_t* __restrict__ idx, int64_t G, Out out) {
  __shared__ uint32_t key[2][kN];
  __shared__ uint32_t words[kN + 4];
  __shared__ int warp_sum[kThreads / 32];
  __shared__ int s_pos, s_has;
  __shared__ double s_gauss;
  const int t = threadIdx.x;
  for (int i = t; i < kN; i += kThreads) key[0][i] = state[i];
  int pos = (int)state[kN];
  int has_gauss = (int)state[kN + 1];
  double gauss = __hiloint2double((int)state[kN + 3], (int)state[kN + 2]);
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

}  // namespace rstart
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_nnd_random_start(uint32_t* state, int64_t n, int32_t k, int32_t d, int32_t* idx, float* P,
                                      int32_t pd1, float* P2, int32_t pd2, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(state && idx, "nnd_random_start: null state or idx");
  UMAPB_REQUIRE(n >= 2 && n - 1 <= 0x7fffffff && k >= 1 && d >= 1, "nnd_random_start: need n >= 2, k >= 1, d >= 1");
  UMAPB_REQUIRE(pd1 >= 0 && pd2 >= 0 && (pd1 == 0 || P) && (pd2 == 0 || P2),
                "nnd_random_start: projection sizes must be >= 0 with their outputs given");
  const uint32_t rng = (uint32_t)(n - 2);  // randint(0, n - 1): values 0 .. n - 2
  uint32_t mask = rng;
  for (int s = 1; s <= 16; s <<= 1) mask |= mask >> s;
  rstart::Out out;
  out.affine = 0;
  out.g1 = (int64_t)d * pd1;
  out.P = P;
  out.s1 = sqrt((double)(pd1 > 0 ? pd1 : 1));
  out.P2 = P2;
  out.s2 = sqrt((double)(pd2 > 0 ? pd2 : 1));
  const int64_t G = out.g1 + (int64_t)d * pd2;
  rstart::random_start_kernel<<<1, rstart::kThreads, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(
      state, k, n * (int64_t)k, rng, mask, idx, G, out);
  UMAPB_LAUNCH_CHECK("nnd_random_start kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_legacy_normal(uint32_t* state, int64_t count, double loc, double scale, float* out,
                                   umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(state && (out || count == 0) && count >= 0, "legacy_normal: bad arguments");
  if (count == 0) return UMAPB_OK;
  rstart::Out o;
  o.affine = 1;
  o.g1 = count;
  o.P = out;
  o.s1 = loc;
  o.P2 = nullptr;
  o.s2 = scale;
  // no bounded integers (count 0): the kernel goes straight to the normals
  rstart::random_start_kernel<<<1, rstart::kThreads, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(
      state, 1, 0, 1u, 1u, nullptr, count, o);
  UMAPB_LAUNCH_CHECK("legacy_normal kernel");
  count_launches(1);
  return UMAPB_OK;
}
