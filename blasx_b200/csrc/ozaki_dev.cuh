// ozaki_dev.cuh -- device code of the emulated GEMM (Ozaki scheme II): the
// CRT constant tables, row statistics, the modulus-count decision, the
// slicing of FP64 / FP32 / complex operands into int8 residues, and the CRT
// reconstruction with the alpha / beta epilogue. Each stage is a device body
// over explicit block coordinates, shared by the standalone kernels
// (ozaki.cu) and the serving executor (executor.cu). Everything here has
// internal linkage: every translation unit that includes it holds its own
// copy of the constant tables and uploads them itself (upload_tables).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "ozaki.h"

namespace bx {
namespace oz {
namespace {

constexpr int kNumN = kMaxModuli - kMinModuli + 1;
// The largest modulus count whose CRT runs on 40-bit FP64 limbs (M < 2^133).
constexpr int kMaxFpCrt = 17;
constexpr int kP = 62;  // |scaled integer| < 2^62

struct CrtTables {
    uint32_t w[kNumN][kMaxModuli][kLimbs];  // CRT weights (M/m_l) * ((M/m_l)^-1 mod m_l)
    uint32_t M[kNumN][kLimbs];              // product of the first N moduli
    double Md[kNumN];                       // M as a double
    double invMd[kNumN];
    int Q[kNumN];                           // norm exponent bound: 2^(2Q) <= M/4
    // the same 32-bit limbs as doubles (exact), operands of the FP64 CRT sums
    // of more than kMaxFpCrt moduli
    double wd[kNumN][kMaxModuli][kLimbs];
    double Ml[kNumN][kLimbs];
    // 40-bit limbs kept at their weight, for up to kMaxFpCrt moduli: limb k
    // of a value v is (bits [40k, 40k + 40) of v) * 2^(40k). wq: the weight
    // limbs times 2^8; cq: their sum over the N moduli; M40: M's limbs.
    double wq[kNumN][kMaxModuli][4];
    double cq[kNumN][4];
    double M40[kNumN][4];
};
__constant__ CrtTables c_crt;

// ---- host bignum helpers (little-endian 32-bit limbs) ----------------------
void big_mul_small(uint32_t *a, int n, uint32_t s) {
    uint64_t carry = 0;
    for (int i = 0; i < n; ++i) {
        uint64_t v = uint64_t(a[i]) * s + carry;
        a[i] = uint32_t(v);
        carry = v >> 32;
    }
}
uint32_t big_div_small(uint32_t *a, int n, uint32_t s) {  // a /= s, returns remainder
    uint64_t rem = 0;
    for (int i = n - 1; i >= 0; --i) {
        uint64_t cur = (rem << 32) | a[i];
        a[i] = uint32_t(cur / s);
        rem = cur % s;
    }
    return uint32_t(rem);
}
// bits [40k, 40k + 40) of a (n 32-bit limbs) times 2^(40k), as an exact double
double limb40(const uint32_t *a, int n, int k, int shift) {
    uint64_t v = 0;
    for (int b = 0; b < 40; ++b) {
        const int bit = 40 * k + b;
        if (bit / 32 < n && ((a[bit / 32] >> (bit % 32)) & 1u)) v |= uint64_t(1) << b;
    }
    return std::ldexp(double(v), 40 * k + shift);
}
double big_to_double(const uint32_t *a, int n) {
    double d = 0;
    for (int i = n - 1; i >= 0; --i) d = d * 4294967296.0 + a[i];
    return d;
}
uint32_t inv_mod(uint32_t a, uint32_t m) {
    for (uint32_t x = 1; x < m; ++x)
        if ((uint64_t(a) * x) % m == 1) return x;
    return 0;
}

CrtTables build_tables() {
    CrtTables t;
    memset(&t, 0, sizeof t);
    for (int n = kMinModuli; n <= kMaxModuli; ++n) {
        const int ni = n - kMinModuli;
        uint32_t M[kLimbs] = {1, 0, 0, 0, 0, 0};
        for (int l = 0; l < n; ++l) big_mul_small(M, kLimbs, uint32_t(kModuli[l]));
        memcpy(t.M[ni], M, sizeof M);
        for (int k = 0; k < kLimbs; ++k) t.Ml[ni][k] = double(M[k]);
        t.Md[ni] = big_to_double(M, kLimbs);
        t.invMd[ni] = 1.0 / t.Md[ni];
        t.Q[ni] = int(std::floor((std::log2(t.Md[ni]) - 2.0) / 2.0));
        for (int l = 0; l < n; ++l) {
            uint32_t q[kLimbs];
            memcpy(q, M, sizeof q);
            big_div_small(q, kLimbs, uint32_t(kModuli[l]));  // M / m_l
            uint32_t tmp[kLimbs];
            memcpy(tmp, q, sizeof tmp);
            const uint32_t r = big_div_small(tmp, kLimbs, uint32_t(kModuli[l]));  // (M/m_l) mod m_l
            big_mul_small(q, kLimbs, inv_mod(r, uint32_t(kModuli[l])));
            memcpy(t.w[ni][l], q, sizeof q);
            for (int k = 0; k < kLimbs; ++k) t.wd[ni][l][k] = double(q[k]);
            for (int k = 0; k < 4; ++k) {
                t.wq[ni][l][k] = limb40(q, kLimbs, k, 8);
                t.cq[ni][k] += t.wq[ni][l][k];  // exact: multiples of 2^(40k+8) below 2^(40k+53)
            }
        }
        for (int k = 0; k < 4; ++k) t.M40[ni][k] = limb40(M, kLimbs, k, 0);
    }
    return t;
}

// ---- device helpers ---------------------------------------------------------

template <typename T> struct Elem;
// cplx: interleaved (re, im) pairs of R; single: the result is rounded to
// FP32 accuracy (u = 2^-24), which sets the modulus count.
template <> struct Elem<double> { static constexpr bool cplx = false, single = false; using R = double; };
template <> struct Elem<float> { static constexpr bool cplx = false, single = true; using R = float; };
struct zpair { double re, im; };
template <> struct Elem<zpair> { static constexpr bool cplx = true, single = false; using R = double; };
struct cpair { float re, im; };
template <> struct Elem<cpair> { static constexpr bool cplx = true, single = true; using R = float; };

// op(X) viewed as R rows x K: element (r, k) at p[k + r*ld] (kc) or p[r + k*ld].
struct View {
    const void *p;
    int64_t ld;
    int64_t R, K;
    int conj;  // negate the imaginary part
};

template <typename T>
__device__ __forceinline__ void load_elem(const View &v, int64_t r, int64_t k, bool kc,
                                          double &re, double &im) {
    const int64_t off = kc ? k + r * v.ld : r + k * v.ld;
    if constexpr (Elem<T>::cplx) {
        using R = typename Elem<T>::R;
        const R *q = static_cast<const R *>(v.p) + 2 * off;
        re = double(q[0]);
        im = v.conj ? -double(q[1]) : double(q[1]);
    } else {
        re = double(static_cast<const T *>(v.p)[off]);
        im = 0.0;
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr), __double_as_longlong(v));
}

// k-contiguous source: one warp per row, lanes stride over k; block bx of
// 256 threads covers rows 8 bx .. 8 bx + 7.
template <typename T>
__device__ __forceinline__ void stats_kc_body(const View &v, const RowStats &st, int64_t bx, int tid) {
    const int64_t r = bx * 8 + (tid >> 5);
    const int lane = tid & 31;
    if (r >= v.R) return;
    double amax = 0, ssq = 0, sab = 0;
    int bad = 0;
    for (int64_t k = lane; k < v.K; k += 32) {
        double re, im;
        load_elem<T>(v, r, k, true, re, im);
        bad |= !(isfinite(re) && isfinite(im));
        const double ar = fabs(re), ai = fabs(im);
        amax = fmax(amax, fmax(ar, ai));
        ssq = fma(re, re, fma(im, im, ssq));
        sab += ar + ai;
    }
    for (int o = 16; o; o >>= 1) {
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        ssq += __shfl_xor_sync(0xffffffffu, ssq, o);
        sab += __shfl_xor_sync(0xffffffffu, sab, o);
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) {
        st.amax[r] = amax;
        st.sumsq[r] = ssq;
        st.sumabs[r] = sab;
        st.flags[r] = bad;
    }
}

// row-contiguous source: one thread per row over a k-chunk, atomics combine;
// block (bx, by) of 256 threads covers rows 256 bx .. 256 bx + 255 and the
// k-chunk by.
template <typename T>
__device__ __forceinline__ void stats_rc_body(const View &v, const RowStats &st, int64_t kchunk, int64_t bx,
                                              int64_t by, int tid) {
    const int64_t r = bx * 256 + tid;
    if (r >= v.R) return;
    const int64_t k0 = by * kchunk, k1 = min(v.K, k0 + kchunk);
    double amax = 0, ssq = 0, sab = 0;
    int bad = 0;
    for (int64_t k = k0; k < k1; ++k) {
        double re, im;
        load_elem<T>(v, r, k, false, re, im);
        bad |= !(isfinite(re) && isfinite(im));
        const double ar = fabs(re), ai = fabs(im);
        amax = fmax(amax, fmax(ar, ai));
        ssq = fma(re, re, fma(im, im, ssq));
        sab += ar + ai;
    }
    atomic_max_nonneg(&st.amax[r], amax);
    atomicAdd(&st.sumsq[r], ssq);
    atomicAdd(&st.sumabs[r], sab);
    if (bad) atomicOr(&st.flags[r], 1);
}

// Chooses the modulus count. Estimated max componentwise error, in units of
// the output dtype's unit roundoff u:
//   E(N) = C * rho_A * rho_B * 2^-q(N) / u,  rho = ||x||_2 sqrt(K) / ||x||_1,
//   q(N) = min(Q_N, P + min_rows log2(||x||_2 / max|x|)),
// calibrated on double-double references (C = 3). The smallest N with
// E(N) <= 1/2 is taken; mode auto falls back to native (N = 0) when even
// kMaxModuli does not reach it, mode ozaki takes kMaxModuli instead.
// One block of nthreads (a multiple of 32, at most 1024) threads.
__device__ __forceinline__ void decide_body(const RowStats &sa, int64_t Ra, const RowStats &sb, int64_t Rb,
                                           int64_t K, double unit, int mode, int forced, Decision *dec, int tid,
                                           int nthreads) {
    __shared__ double s_rho[2][32], s_h[2][32];
    __shared__ int s_bad[32];
    double rho[2] = {0, 0}, h[2] = {1e300, 1e300};
    int bad = 0;
    for (int side = 0; side < 2; ++side) {
        const RowStats &st = side ? sb : sa;
        const int64_t R = side ? Rb : Ra;
        for (int64_t r = tid; r < R; r += nthreads) {
            bad |= st.flags[r];
            const double n1 = st.sumabs[r];
            if (n1 > 0) {
                const double n2 = sqrt(st.sumsq[r]);
                rho[side] = fmax(rho[side], n2 * sqrt(double(K)) / n1);
                h[side] = fmin(h[side], log2(n2 / st.amax[r]));
            }
        }
    }
    const int lane = tid & 31, w = tid >> 5;
    for (int o = 16; o; o >>= 1) {
        for (int sd = 0; sd < 2; ++sd) {
            rho[sd] = fmax(rho[sd], __shfl_xor_sync(0xffffffffu, rho[sd], o));
            h[sd] = fmin(h[sd], __shfl_xor_sync(0xffffffffu, h[sd], o));
        }
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) {
        s_rho[0][w] = rho[0]; s_rho[1][w] = rho[1];
        s_h[0][w] = h[0]; s_h[1][w] = h[1];
        s_bad[w] = bad;
    }
    __syncthreads();
    if (tid != 0) return;
    const int nw = nthreads / 32;
    for (int i = 1; i < nw; ++i) {
        for (int sd = 0; sd < 2; ++sd) {
            s_rho[sd][0] = fmax(s_rho[sd][0], s_rho[sd][i]);
            s_h[sd][0] = fmin(s_h[sd][0], s_h[sd][i]);
        }
        s_bad[0] |= s_bad[i];
    }
    Decision d;
    d.nonfinite = s_bad[0];
    d.pad = 0;
    const double ra = fmax(s_rho[0][0], 1.0), rb = fmax(s_rho[1][0], 1.0);
    const double ha = s_h[0][0] > 1e299 ? 0.0 : s_h[0][0];
    const double hb = s_h[1][0] > 1e299 ? 0.0 : s_h[1][0];
    int chosen = 0;
    double est = 0;
    for (int n = kMinModuli; n <= kMaxModuli; ++n) {
        const int ni = n - kMinModuli;
        const double qa = fmin(double(c_crt.Q[ni]), kP + ha);
        const double qb = fmin(double(c_crt.Q[ni]), kP + hb);
        est = 3.0 * ra * rb * exp2(-fmin(qa, qb)) / unit;
        if (forced ? n == forced : est <= 0.5) {
            chosen = n;
            break;
        }
    }
    if (!chosen && mode == 2) chosen = kMaxModuli;
    if (d.nonfinite) chosen = 0;  // Inf/NaN: the native kernel propagates them
    d.nmod = chosen;
    d.q = chosen ? c_crt.Q[chosen - kMinModuli] : 0;
    d.estimate = est;
    *dec = d;
}

// Row exponent: 2^e ||x||_2 < 2^Q and 2^e max|x| < 2^P. When the sum of
// squares over- or underflowed, ||x||_2 <= max|x| sqrt(K) is used instead.
__device__ __forceinline__ int row_exponent(double amax, double sumsq, int Q, int64_t K) {
    if (!(amax > 0)) return 0;
    double n2 = sqrt(sumsq);
    if (!(n2 >= amax) || !isfinite(n2)) n2 = amax * sqrt(double(K)) * 2.0;
    const int en = Q - 1 - ilogb(n2);
    const int em = kP - 1 - ilogb(amax);
    return min(en, em);
}

// The moduli as compile-time constants for the device code (same order as
// kModuli). Every helper below takes the modulus index as a template
// parameter, so the per-modulus constants fold at compile time whatever the
// unrolling decisions of the compiler.
template <int L> struct Mod {
    static_assert(L >= 0 && L < kMaxModuli, "modulus index");
    static constexpr uint32_t table[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239,
                                                   233, 229, 227, 223, 217, 211, 199,
                                                   197, 193, 191, 181, 179, 173};
    static constexpr uint32_t m = table[L];
    static constexpr uint32_t pw(int bits) { return uint32_t((uint64_t(1) << bits) % m); }
    // 2^(8k) mod m, one byte each: bytes 0-3 of the biased value (lo) and
    // bytes 4-7 (hi)
    static constexpr uint32_t wlo = pw(0) | pw(8) << 8 | pw(16) << 16 | pw(24) << 24;
    static constexpr uint32_t whi = pw(32) | pw(40) << 8 | pw(48) << 16 | pw(56) << 24;
    // half range of the symmetric residue (m odd): [-h, h]
    static constexpr uint32_t h = (m - 1) / 2;
    // -2^62 mod m: removes the bias
    static constexpr uint32_t cb = uint32_t((m - (uint64_t(1) << 62) % m) % m);
    // ceil(2^32 / m): the quotient of t < 2^20 by m is its product's high word
    static constexpr uint32_t magic = uint32_t(((uint64_t(1) << 32) + m - 1) / m);
    // h * magic: (s + h) * magic as one 64-bit multiply-add of s
    static constexpr uint64_t hmagic = uint64_t(h) * magic;
};

// v + 2^62 (|v| < 2^62, so the biased value is in [0, 2^63)) as two 32-bit
// words, computed once per element and shared by all moduli.
struct Digits {
    uint32_t lo, hi;
};
__device__ __forceinline__ Digits digits_of(int64_t v) {
    const uint64_t a = uint64_t(v) + (uint64_t(1) << 62);
    return {uint32_t(a), uint32_t(a >> 32)};
}

// Symmetric residue of v for the L-th modulus, in [-h, h] for odd m (the
// low byte for m = 256, whose byte is already the two's complement of the
// residue in [-128, 127]): with the bias removed, the bytes b_k of the
// biased value give
//   s = sum_k b_k (2^(8k) mod m) + (-2^62 mod m) <= 8 * 255 * 255 + 255,
// two byte dot products (DP4A) against constant weight words, s = v (mod m).
// With t = s + h < 2^20,
//   q = floor(t / m) = floor(t ceil(2^32/m) / 2^32), exact for t < 2^20 and
// m <= 256 (the rounding error of the magic multiplier, below 2^-12, stays
// under 1/m), is the high word of s * magic + h * magic, and
// s - q m = (v + h) mod m - h is the residue of v in [-h, h]. Every constant
// folds: two DP4As, one wide multiply-add, one IMAD.
template <int L> __device__ __forceinline__ int32_t residue_s(const Digits &x) {
    using C = Mod<L>;
    if constexpr (C::m == 256) {
        return int32_t(x.lo);
    } else {
        const uint32_t s = __dp4a(x.hi, C::whi, __dp4a(x.lo, C::wlo, C::cb));
        const uint32_t q = uint32_t((uint64_t(s) * C::magic + C::hmagic) >> 32);
        return int32_t(s - q * C::m);
    }
}

// The low bytes of four values packed into one word (byte k from value k).
__device__ __forceinline__ uint32_t pack_bytes(int32_t a, int32_t b, int32_t c, int32_t d) {
    return __byte_perm(__byte_perm(uint32_t(a), uint32_t(b), 0x0040u),
                       __byte_perm(uint32_t(c), uint32_t(d), 0x0040u), 0x5410u);
}

// x * 2^e for a normal x: one multiply by a constructed power of two when
// 2^e is a normal double, ldexp otherwise (both round the same way).
__device__ __forceinline__ double scale_pow2(double x, int e) {
    if (e >= -1022 && e <= 1023) return x * __longlong_as_double(int64_t(e + 1023) << 52);
    return ldexp(x, e);
}

__device__ __forceinline__ int64_t scale_round(double x, int e) {
    return __double2ll_rn(scale_pow2(x, e));
}

// Output geometry of one operand's slices.
//   role 0 (real):      out[l][r][k]
//   role 1 (complex Y): out[l][r][k] = re, out[l][r][Kh + k] = im
//   role 2 (complex X): out[l][r][k] = re, out[l][r][Kh+k] = -im,
//                       out[l][Rp + r][k] = im, out[l][Rp + r][Kh + k] = re
struct SliceOut {
    int8_t *p;
    int64_t Rp;      // padded rows of one block
    int64_t Kp;      // row length (bytes)
    int64_t Kh;      // complex half length (0 for real)
    int64_t plane;   // bytes per modulus plane
};

// Packs the symmetric residues of 16 consecutive elements for modulus L.
template <int L> __device__ __forceinline__ uint4 pack16(const Digits (&x)[16]) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        w[q] = pack_bytes(residue_s<L>(x[4 * q]), residue_s<L>(x[4 * q + 1]), residue_s<L>(x[4 * q + 2]),
                          residue_s<L>(x[4 * q + 3]));
    return make_uint4(w[0], w[1], w[2], w[3]);
}
__device__ __forceinline__ uint4 neg16(uint4 a) {  // residue of -x, byte-wise
    return make_uint4(__vneg4(a.x), __vneg4(a.y), __vneg4(a.z), __vneg4(a.w));
}

// Writes the residues, for modulus L, of component COMP (0 re, 1 im) of 16
// consecutive k (k0 multiple of 16) of row r, to every place the role puts
// that component.
template <int ROLE, int COMP, int L>
__device__ __forceinline__ void store16(const SliceOut &o, int64_t r, int64_t k0,
                                        const Digits (&x)[16]) {
    int8_t *base = o.p + int64_t(L) * o.plane;
    const uint4 w = pack16<L>(x);
    if (COMP == 0) {
        *reinterpret_cast<uint4 *>(base + r * o.Kp + k0) = w;
        if (ROLE == 2) *reinterpret_cast<uint4 *>(base + (o.Rp + r) * o.Kp + o.Kh + k0) = w;
    } else if (ROLE == 1) {
        *reinterpret_cast<uint4 *>(base + r * o.Kp + o.Kh + k0) = w;
    } else if (ROLE == 2) {
        *reinterpret_cast<uint4 *>(base + r * o.Kp + o.Kh + k0) = neg16(w);
        *reinterpret_cast<uint4 *>(base + (o.Rp + r) * o.Kp + k0) = w;
    }
}

// Moduli L, L+1, ..., nmod-1 by compile-time recursion.
template <int ROLE, int COMP, int L = 0>
__device__ __forceinline__ void store_all(const SliceOut &o, int nmod, int64_t r, int64_t k0,
                                          const Digits (&x)[16]) {
    if constexpr (L < kMaxModuli) {
        if (L < nmod) {
            store16<ROLE, COMP, L>(o, r, k0, x);
            store_all<ROLE, COMP, L + 1>(o, nmod, r, k0, x);
        }
    }
}

// k-contiguous source: a thread scales 16 consecutive k of one row and
// writes one 16-byte word per modulus (and place), one component at a time
// (the second pass re-reads the same 16-byte elements, from L1).
// grid (Kc/64, Rp/64), block 256: row = tid / 4, k = 16 (tid % 4).
template <typename T, int ROLE, int COMP>
__device__ __forceinline__ void slice_kc_comp(const View &v, int nmod, int e, int64_t r, int64_t k0,
                                              const SliceOut &o) {
    Digits d[16];
    bool done = false;
    if constexpr (!Elem<T>::cplx) {
        // 16 whole elements in range and 16-byte aligned: vector loads
        const T *p = static_cast<const T *>(v.p) + (r * v.ld + k0);
        if (r < v.R && k0 + 16 <= v.K && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
            constexpr int PER = 16 / sizeof(T);  // elements per 16-byte load
            using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
            T x[16];
#pragma unroll
            for (int q = 0; q < 16; q += PER) *reinterpret_cast<V *>(&x[q]) = __ldcg(reinterpret_cast<const V *>(p + q));
#pragma unroll
            for (int q = 0; q < 16; ++q) d[q] = digits_of(scale_round(double(x[q]), e));
            done = true;
        }
    }
    if (!done) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            double re = 0, im = 0;
            if (r < v.R && k0 + q < v.K) load_elem<T>(v, r, k0 + q, true, re, im);
            d[q] = digits_of(scale_round(COMP ? im : re, e));
        }
    }
    store_all<ROLE, COMP>(o, nmod, r, k0, d);
}

template <typename T, int ROLE>
__device__ __forceinline__ void slice_kc_body(const View &v, const RowStats &st, const Decision *dec, int *expo,
                                              const SliceOut &o, int64_t bx, int64_t by, int tid) {
    const int nmod = dec->nmod;
    if (nmod == 0) return;
    const int Q = dec->q;
    const int64_t r = by * 64 + (tid >> 2);
    const int64_t k0 = bx * 64 + (tid & 3) * 16;
    int e = 0;
    if (r < v.R) e = row_exponent(st.amax[r], st.sumsq[r], Q, v.K);
    if (bx == 0 && (tid & 3) == 0 && r < v.R) expo[r] = e;
    slice_kc_comp<T, ROLE, 0>(v, nmod, e, r, k0, o);
    if (ROLE) slice_kc_comp<T, ROLE, 1>(v, nmod, e, r, k0, o);
}

// row-contiguous source: a 64-row x KT-k tile is read along rows, scaled,
// and its integers are transposed once through shared memory; then a thread
// owns 16 consecutive k of one row and one component, as in the
// k-contiguous kernel (complex: warps 0-3 the real parts, 4-7 the imaginary).
// grid (Kc/KT, Rp/64), block 256; smem holds slice_rc_smem_bytes<ROLE>()
// bytes (the transposed tile, then the 64 row exponents).
template <int ROLE> constexpr size_t slice_rc_smem_bytes() {
    return size_t(ROLE ? 2 : 1) * (ROLE ? 32 : 64) * (64 + 1) * sizeof(int64_t) + 64 * sizeof(int);
}
template <typename T, int ROLE>
__device__ __forceinline__ void slice_rc_body(const View &v, const RowStats &st, const Decision *dec, int *expo,
                                              const SliceOut &o, int64_t bx, int64_t by, int tid, void *smem) {
    constexpr int KT = ROLE ? 32 : 64;
    constexpr int CPL = ROLE ? 2 : 1;
    int64_t (*tile)[KT][64 + 1] = reinterpret_cast<int64_t (*)[KT][64 + 1]>(smem);
    int *s_e = reinterpret_cast<int *>(static_cast<char *>(smem) + size_t(CPL) * KT * (64 + 1) * sizeof(int64_t));
    const int nmod = dec->nmod;
    if (nmod == 0) return;
    const int Q = dec->q;
    const int64_t r0 = by * 64, k0 = bx * KT;
    if (tid < 64) {
        const int64_t r = r0 + tid;
        int e = 0;
        if (r < v.R) e = row_exponent(st.amax[r], st.sumsq[r], Q, v.K);
        s_e[tid] = e;
        if (bx == 0 && r < v.R) expo[r] = e;
    }
    __syncthreads();
    bool paired = false;
    if constexpr (std::is_same<T, double>::value) {
        // FP64 rows in pairs: one 16-byte load covers rows r, r + 1 of one k
        // (ld even, 16-byte aligned base; the block's first row is even)
        const double *p = static_cast<const double *>(v.p);
        if ((v.ld & 1) == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
            paired = true;
            const int tr = (tid & 31) * 2, tk = tid >> 5;  // tk in 0..7
            const int64_t r = r0 + tr;
            const int e0 = s_e[tr], e1 = s_e[tr + 1];
#pragma unroll
            for (int i = 0; i < KT / 8; ++i) {
                const int kk = tk + 8 * i;
                double2 x = make_double2(0.0, 0.0);
                if (k0 + kk < v.K) {
                    const double *q = p + r + (k0 + kk) * v.ld;
                    if (r + 1 < v.R) x = __ldcg(reinterpret_cast<const double2 *>(q));
                    else if (r < v.R) x.x = q[0];
                }
                tile[0][kk][tr] = scale_round(x.x, e0);
                tile[0][kk][tr + 1] = scale_round(x.y, e1);
            }
        }
    }
    if (!paired) {
        const int tr = tid & 63, tk = tid >> 6;  // tk in 0..3
        const int64_t r = r0 + tr;
        const int e = s_e[tr];
#pragma unroll
        for (int i = 0; i < KT / 4; ++i) {
            const int kk = tk + 4 * i;
            double re = 0, im = 0;
            if (r < v.R && k0 + kk < v.K) load_elem<T>(v, r, k0 + kk, false, re, im);
            tile[0][kk][tr] = scale_round(re, e);
            if (ROLE) tile[CPL - 1][kk][tr] = scale_round(im, e);
        }
    }
    __syncthreads();
    constexpr int TPR = KT / 16;  // threads per row and component
    static_assert(64 * TPR * CPL == 256, "one 16-k word per thread");
    // a warp reads 32 consecutive rows of one k-group: conflict-free
    const int comp = tid / (64 * TPR), idx = tid % (64 * TPR);
    const int wr = idx % 64, wk = (idx / 64) * 16;
    Digits d[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) d[q] = digits_of(tile[comp][wk + q][wr]);
    if (comp == 0) store_all<ROLE, 0>(o, nmod, r0 + wr, k0 + wk, d);
    else if (ROLE) store_all<ROLE, 1>(o, nmod, r0 + wr, k0 + wk, d);
}

// ---- reconstruction -----------------------------------------------------------

// 32-bit limbs that hold the weights w_l < M and M itself for N moduli; the
// signed result |X| < M/4 then fits with its sign bit.
__host__ __device__ constexpr int limbs_for(int n) {
    return n <= 8 ? 2 : n <= 12 ? 3 : n <= 16 ? 4 : 5;
}

// Residue l of element qb (byte qb of w[l], in [0, 256)) as an exact double:
// the byte is placed in the low mantissa bits of 2^52 and 2^52 taken off.
__device__ __forceinline__ double residue_as_double(uint32_t w, int qb) {
    return __hiloint2double(0x43300000, int(__byte_perm(w, 0u, 0x4440u | uint32_t(qb)))) -
           4503599627370496.0;
}

// 1 + u / 256 for the residue u = byte qb of w: exact (9 significant bits),
// built in the high word alone.
__device__ __forceinline__ double residue_plus_one(uint32_t w, int qb) {
    const uint32_t u = __byte_perm(w, 0u, 0x4440u | uint32_t(qb));
    return __hiloint2double(int(u * 4096u + 0x3FF00000u), 0);
}

// s + e = a + b exactly (Knuth's TwoSum).
__device__ __forceinline__ double two_sum(double a, double b, double &e) {
    const double s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return s;
}

// a + b rounded to odd: the truncation of the exact sum, its last mantissa
// bit set when the sum is inexact (the neighbour of the round-to-nearest
// result toward the exact sum, when that result's last bit is even).
__device__ __forceinline__ double add_round_odd(double a, double b) {
    double e;
    const double s = two_sum(a, b, e);
    long long bits = __double_as_longlong(s);
    if (e != 0.0 && !(bits & 1)) bits += ((e > 0.0) == (s > 0.0)) ? 1 : -1;
    return __longlong_as_double(bits);
}

// The CRT value of one entry's residues times 2^scale as a double,
// correctly rounded from the exact integer X (the scaling by a power of two
// is exact unless the result leaves the normal range):
//   S = sum_l u_l w_l is congruent to X mod M, and the row and column
//   scaling guarantees |X| < 2^(2Q) <= M/4. X = S - q M with q = rint(S / M):
//   S / M lies within 1/4 of an integer and its double estimate is off by
//   far less, so the rounding is never ambiguous.
// Up to kMaxFpCrt moduli (M < 2^133) everything runs on the FP64 pipe. With
// w_l and M cut into L limbs of 40 bits kept at their weight 2^(40k), every
// limb sum S_k = sum_l u_l w_{l,k} is a multiple of 2^(40k) below
// 2^(40k+53): exact. It is accumulated as sum_l (1 + u_l/256) (256 w_{l,k})
// from -sum_l 256 w_{l,k}, each product exact (9 x 40 significant bits) and
// each partial sum exact, so the residue enters as a bit pattern, without a
// conversion. The differences D_k = S_k - q M_k (|D_k| < 2^(40k+53), one
// DFMA each) are exact, and X = D_0 + D_1 + D_2 (with D_3 + D_2, exact since
// |X| < 2^131, as the top term for four limbs). The sum of the three is
// rounded correctly by the round-to-odd method of Boldo and Melquiond
// ("Emulation of FMA and correctly rounded sums: proved algorithms using
// rounding to odd", IEEE Trans. Computers 57(4), 2008):
//   (uh, ul) = TwoSum(D_1, D_0), (th, tl) = TwoSum(D_2, uh),
//   RN(X) = RN(th + RO(tl + ul)).
// More moduli use 32-bit limbs: D_t = S_t - q M_t with |D_t| < 2^45, whose
// two's complement words come out of the mantissa of D_t + 1.5 * 2^52; a
// carry pass assembles X in L words, and its magnitude is converted with one
// rounding from a 64-bit window and a sticky bit.

// 40-bit limbs of M for the FP64 CRT of N <= kMaxFpCrt moduli.
template <int N> __host__ __device__ constexpr int fp_limbs() { return N <= 10 ? 2 : N <= 15 ? 3 : 4; }

// The FP64 CRT's limb sums S_k of the 4 rows whose residues w packs (byte q
// of w[l]: row q, modulus l), all rows at once: every weight limb is read once
// and serves the 4 rows.
template <int N>
__device__ __forceinline__ void crt_sums4(const uint32_t (&w)[N], double (&S)[4][fp_limbs<N>()]) {
    constexpr int L = fp_limbs<N>(), ni = N - kMinModuli;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int k = 0; k < L; ++k) S[q][k] = -c_crt.cq[ni][k];
#pragma unroll
    for (int l = 0; l < N; ++l) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double d = residue_plus_one(w[l], q);
#pragma unroll
            for (int k = 0; k < L; ++k) S[q][k] = __fma_rn(d, c_crt.wq[ni][l][k], S[q][k]);
        }
    }
}

// RN(X) * 2^scale from one row's limb sums (N <= kMaxFpCrt).
template <int N>
__device__ __forceinline__ double crt_round(const double (&S)[fp_limbs<N>()], int scale) {
    constexpr int L = fp_limbs<N>(), ni = N - kMinModuli;
    const double qd = rint(__dmul_rn(__dadd_rn(S[L - 1], S[L - 2]), c_crt.invMd[ni]));
    double D[L];
#pragma unroll
    for (int k = 0; k < L; ++k) D[k] = __fma_rn(-qd, c_crt.M40[ni][k], S[k]);
    double x;
    if constexpr (L == 2) {
        x = __dadd_rn(D[1], D[0]);
    } else {
        const double top = L == 4 ? __dadd_rn(D[3], D[2]) : D[2];
        double ul, tl;
        const double uh = two_sum(D[1], D[0], ul);
        const double th = two_sum(top, uh, tl);
        x = __dadd_rn(th, add_round_odd(tl, ul));
    }
    return scale_pow2(__dadd_rn(x, 0.0), scale);  // + 0: a zero sum is +0
}

// CRT of more than kMaxFpCrt moduli for row qb of w (the 32-bit-limb method).
// Out of line: its registers would otherwise size every reconstruction
// kernel, whose common path (fewer moduli) needs far fewer.
template <int N>
__device__ __noinline__ double crt_to_double(const uint32_t (&w)[N], int qb, int scale) {
    constexpr int ni = N - kMinModuli;
    static_assert(N > kMaxFpCrt, "the FP64-limb CRT serves fewer moduli");
    {
        constexpr int L = limbs_for(N);
        double S[L];
#pragma unroll
        for (int t = 0; t < L; ++t) S[t] = 0.0;
#pragma unroll
        for (int l = 0; l < N; ++l) {
            const double u = residue_as_double(w[l], qb);
#pragma unroll
            for (int t = 0; t < L; ++t) S[t] = fma(u, c_crt.wd[ni][l][t], S[t]);
        }
        double sa = S[L - 1];
#pragma unroll
        for (int t = L - 2; t >= 0; --t) sa = fma(sa, 4294967296.0, S[t]);
        const double qd = rint(sa * c_crt.invMd[ni]);
        uint32_t x[L];
        int32_t carry = 0;
#pragma unroll
        for (int t = 0; t < L; ++t) {
            const double d = fma(-qd, c_crt.Ml[ni][t], S[t]) + 6755399441055744.0;
            const uint32_t lo = uint32_t(__double2loint(d));
            const int32_t hi = __double2hiint(d) - 0x43380000;
            const int64_t v = int64_t(lo) + int64_t(carry);
            x[t] = uint32_t(v);
            carry = hi + int32_t(v >> 32);  // floor division: -1, 0 or 1 from the low word
        }
        const bool neg = int32_t(x[L - 1]) < 0;
        if (neg) {  // magnitude: ~x + 1
            uint32_t c = 1;
#pragma unroll
            for (int t = 0; t < L; ++t) {
                const uint64_t v = uint64_t(~x[t]) + c;
                x[t] = uint32_t(v);
                c = uint32_t(v >> 32);
            }
        }
        // magnitude -> double, correctly rounded: a 64-bit window whose bit
        // 63 is the leading one, every lower bit folded into a sticky bit 0
        // (bit 0 lies below the 53-bit rounding point, so round-to-nearest-
        // even stays exact)
        int top = -1;
#pragma unroll
        for (int t = L - 1; t >= 0; --t)
            if (top < 0 && x[t]) top = t;
        if (top < 0) return 0.0;
        uint32_t xt = 0, xt1 = 0, xt2 = 0, sticky = 0;
#pragma unroll
        for (int t = 0; t < L; ++t) {
            if (t == top) xt = x[t];
            if (t == top - 1) xt1 = x[t];
            if (t == top - 2) xt2 = x[t];
            if (t < top - 2) sticky |= x[t];
        }
        const uint64_t hi64 = (uint64_t(xt) << 32) | xt1;
        const int lz = __clzll(hi64);  // < 32 because xt != 0
        uint64_t win = hi64 << lz;
        if (lz) {
            win |= uint64_t(xt2) >> (32 - lz);
            sticky |= xt2 << lz;
        } else {
            sticky |= xt2;
        }
        if (sticky) win |= 1;
        const double d = scale_pow2(__ull2double_rn(win), 32 * (top - 1) - lz + scale);
        return neg ? -d : d;
    }
}

// Gathers 4 consecutive rows' residues of one column: w[l] packs the uint8
// residues of rows i0..i0+3 for modulus l.
template <int N>
__device__ __forceinline__ void gather4(const uint8_t *U, int64_t plane, int64_t row_off,
                                        uint32_t (&w)[N]) {
#pragma unroll
    for (int l = 0; l < N; ++l) w[l] = *reinterpret_cast<const uint32_t *>(U + l * plane + row_off);
}

struct ReconArgs {
    const uint8_t *U;
    int64_t Jp, Ip, M, N;
    const int *ea, *fb;
    double ar, ai, br, bi;
    int beta_zero;
    void *C;
    int64_t ldc;
    int64_t j0;  // first column of this launch
    int uplo;    // triangular output: 0 all, 1 i - j <= diag, 2 i - j >= diag
    int64_t diag;
};

__device__ __forceinline__ bool recon_keep(const ReconArgs &a, int64_t i, int64_t j) {
    return a.uplo == 0 || (a.uplo == 1 ? i - j <= a.diag : i - j >= a.diag);
}

template <typename T, int N>
__device__ __forceinline__ void recon_real(const ReconArgs &a, int64_t i0, int64_t j) {
    uint32_t w[N];
    gather4<N>(a.U, a.Jp * a.Ip, j * a.Ip + i0, w);
    const int fj = a.fb[j];
    T *C = static_cast<T *>(a.C);
    auto put = [&](int64_t i, double val) {
        T *cp = C + i + j * a.ldc;
        double r = a.ar * val;
        if (!a.beta_zero) r = fma(a.br, double(*cp), r);
        *cp = T(r);
    };
    if constexpr (N <= kMaxFpCrt) {
        double S[4][fp_limbs<N>()];
        crt_sums4<N>(w, S);
        T *cp = C + i0 + j * a.ldc;
        if (a.uplo == 0 && i0 + 3 < a.M && (reinterpret_cast<uintptr_t>(cp) & 15) == 0) {
            // 4 whole rows, 16-byte aligned: vector loads and stores of C and
            // the row exponents, the same arithmetic per entry as put
            const int4 e = *reinterpret_cast<const int4 *>(a.ea + i0);
            double r[4] = {crt_round<N>(S[0], -(e.x + fj)), crt_round<N>(S[1], -(e.y + fj)),
                           crt_round<N>(S[2], -(e.z + fj)), crt_round<N>(S[3], -(e.w + fj))};
#pragma unroll
            for (int q = 0; q < 4; ++q) r[q] = a.ar * r[q];
            if constexpr (std::is_same<T, double>::value) {
                double2 *v = reinterpret_cast<double2 *>(cp);
                if (!a.beta_zero) {
                    const double2 c0 = v[0], c1 = v[1];
                    r[0] = fma(a.br, c0.x, r[0]);
                    r[1] = fma(a.br, c0.y, r[1]);
                    r[2] = fma(a.br, c1.x, r[2]);
                    r[3] = fma(a.br, c1.y, r[3]);
                }
                v[0] = make_double2(r[0], r[1]);
                v[1] = make_double2(r[2], r[3]);
            } else {
                float4 *v = reinterpret_cast<float4 *>(cp);
                if (!a.beta_zero) {
                    const float4 c = *v;
                    r[0] = fma(a.br, double(c.x), r[0]);
                    r[1] = fma(a.br, double(c.y), r[1]);
                    r[2] = fma(a.br, double(c.z), r[2]);
                    r[3] = fma(a.br, double(c.w), r[3]);
                }
                *v = make_float4(float(r[0]), float(r[1]), float(r[2]), float(r[3]));
            }
            return;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t i = i0 + q;
            if (i < a.M && recon_keep(a, i, j)) put(i, crt_round<N>(S[q], -(a.ea[i] + fj)));
        }
    } else {
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
            const int64_t i = i0 + q;
            if (i >= a.M) break;
            if (!recon_keep(a, i, j)) continue;
            put(i, crt_to_double<N>(w, q, -(a.ea[i] + fj)));
        }
    }
}

template <typename T, int N>
__device__ __forceinline__ void recon_cplx(const ReconArgs &a, int64_t i0, int64_t j) {
    using R = typename Elem<T>::R;
    const int64_t plane = 2 * a.Jp * a.Ip;
    uint32_t wr[N], wi[N];
    gather4<N>(a.U, plane, j * a.Ip + i0, wr);
    gather4<N>(a.U, plane, (a.Jp + j) * a.Ip + i0, wi);
    const int fj = a.fb[j];
    R *C = static_cast<R *>(a.C);
    // one entry: (re, im) loaded and stored as one vector (16 bytes for
    // complex128, 8 for complex64) when C is aligned to that size
    using V = typename std::conditional<std::is_same<R, double>::value, double2, float2>::type;
    const bool vec = (reinterpret_cast<uintptr_t>(a.C) & (sizeof(V) - 1)) == 0;
    auto put = [&](int64_t i, double xr, double xi) {
        R *cp = C + 2 * (i + j * a.ldc);
        double vr = a.ar * xr - a.ai * xi, vi = a.ar * xi + a.ai * xr;
        if (vec) {
            V *vp = reinterpret_cast<V *>(cp);
            if (!a.beta_zero) {
                const V c = *vp;
                const double cr = double(c.x), ci = double(c.y);
                vr += a.br * cr - a.bi * ci;
                vi += a.br * ci + a.bi * cr;
            }
            V o;
            o.x = R(vr);
            o.y = R(vi);
            *vp = o;
        } else {
            if (!a.beta_zero) {
                const double cr = double(cp[0]), ci = double(cp[1]);
                vr += a.br * cr - a.bi * ci;
                vi += a.br * ci + a.bi * cr;
            }
            cp[0] = R(vr);
            cp[1] = R(vi);
        }
    };
    if constexpr (N <= kMaxFpCrt) {
        // the real parts of the 4 rows, then the imaginary parts
        double xr[4], S[4][fp_limbs<N>()];
        int sc[4];
        bool live[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t i = i0 + q;
            live[q] = i < a.M && recon_keep(a, i, j);
            sc[q] = live[q] ? -(a.ea[i] + fj) : 0;
        }
        crt_sums4<N>(wr, S);
#pragma unroll
        for (int q = 0; q < 4; ++q) xr[q] = crt_round<N>(S[q], sc[q]);
        crt_sums4<N>(wi, S);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (live[q]) put(i0 + q, xr[q], crt_round<N>(S[q], sc[q]));
    } else {
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
            const int64_t i = i0 + q;
            if (i >= a.M) break;
            if (!recon_keep(a, i, j)) continue;
            const int sc = -(a.ea[i] + fj);
            put(i, crt_to_double<N>(wr, q, sc), crt_to_double<N>(wi, q, sc));
        }
    }
}

// One thread per 4 consecutive rows i of a column j. The modulus count is
// read on the device; the switch is uniform, each case fully unrolled.
// Block (bx, by) of 128 threads: column j0 + by, rows 512 bx .. 512 bx + 511.
template <typename T, bool CPLX>
__device__ __forceinline__ void reconstruct_body(const ReconArgs &a, const Decision *dec, int64_t bx, int64_t by,
                                                 int tid) {
    const int n = dec->nmod;
    if (n == 0) return;
    const int64_t j = a.j0 + by;
    const int64_t i0 = (bx * 128 + tid) * 4;
    if (i0 >= a.M || j >= a.N) return;
#define BX_RECON_CASE(NN)                                     \
    case NN:                                                  \
        if constexpr (CPLX) recon_cplx<T, NN>(a, i0, j);      \
        else recon_real<T, NN>(a, i0, j);                     \
        break;
    switch (n) {
        BX_RECON_CASE(6) BX_RECON_CASE(7) BX_RECON_CASE(8) BX_RECON_CASE(9) BX_RECON_CASE(10)
        BX_RECON_CASE(11) BX_RECON_CASE(12) BX_RECON_CASE(13) BX_RECON_CASE(14)
        BX_RECON_CASE(15) BX_RECON_CASE(16) BX_RECON_CASE(17) BX_RECON_CASE(18)
        BX_RECON_CASE(19) BX_RECON_CASE(20)
        default: break;
    }
#undef BX_RECON_CASE
}


// ---- scratch layout of one emulated GEMM (host) ----------------------------------

struct Carve {
    char *base;
    size_t off = 0;
    template <typename T> T *take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T *p = reinterpret_cast<T *>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

int forced_moduli() {
    static const int f = [] {
        const char *e = getenv("BLASX_OZAKI_MODULI");
        const int v = e ? atoi(e) : 0;
        return (v >= kMinModuli && v <= kMaxModuli) ? v : 0;
    }();
    return f;
}

// Padded extents and scratch size of one emulated GEMM.
struct Plan {
    int64_t M, N, K, Kh, Kp, Kc, Ip, Jp, Jx;
    bool alias;  // op(B) = op(A)^T on the same buffer (SYRK): X is Y, sliced once
    size_t bytes;
};

// op(B) = op(A)^T read from the same buffer (real types): the rows of op(A)
// are the columns of op(B), so their statistics, exponents and slices agree.
bool aliased(const Gemm &g) {
    return !is_complex(g.dt) && g.A == g.B && g.lda == g.ldb && g.M == g.N &&
           (g.ta == NoTrans) != (g.tb == NoTrans);
}

Plan make_plan(const Gemm &g) {
    const bool cplx = is_complex(g.dt);
    const int64_t L = kMaxModuli;
    Plan p;
    p.M = g.M; p.N = g.N; p.K = g.K;
    p.Kh = cplx ? pad(p.K, 64) : 0;
    p.Kp = cplx ? 2 * p.Kh : pad(p.K, kTileK);
    p.Kc = cplx ? p.Kh : p.Kp;  // k extent covered by the slice kernels
    p.Ip = pad(p.M, kTileI);
    p.alias = aliased(g);
    p.Jp = p.alias ? p.Ip : pad(p.N, kTileJ);
    p.Jx = cplx ? 2 * p.Jp : p.Jp;  // X rows (Re block + Im block)
    p.bytes = 256 * 16 + (3 * sizeof(double) + 2 * sizeof(int)) * size_t(p.M + p.N) +
              sizeof(Decision) + sizeof(int) + size_t(L) * p.Ip * p.Kp +
              (p.alias ? 0 : size_t(L) * p.Jx * p.Kp) + size_t(L) * p.Jx * p.Ip;
    return p;
}


// Device pointers of one emulated GEMM's scratch (make_plan(g).bytes bytes at
// ws). The error word comes first: the same offset for every shape, so a
// sequence of steps on one scratch accumulates into one word.
struct Parts {
    int *err;
    Decision *dec;
    RowStats sa, sb;
    int *ea, *fb;
    int8_t *Y, *X;
    uint8_t *U;
    size_t stats_bytes;  // sa and sb, contiguous from sa.amax: cleared before the statistics
};
inline Parts carve_parts(const Gemm &g, const Plan &pl, void *ws) {
    const int64_t L = kMaxModuli;
    Carve cv{static_cast<char *>(ws)};
    Parts p;
    p.err = cv.take<int>(1);
    p.dec = cv.take<Decision>(1);
    p.sa = RowStats{cv.take<double>(pl.M), cv.take<double>(pl.M), cv.take<double>(pl.M), cv.take<int>(pl.M)};
    p.sb = RowStats{cv.take<double>(pl.N), cv.take<double>(pl.N), cv.take<double>(pl.N), cv.take<int>(pl.N)};
    p.ea = cv.take<int>(pl.M);
    p.fb = cv.take<int>(pl.N);
    p.Y = cv.take<int8_t>(size_t(L) * pl.Ip * pl.Kp);
    p.X = pl.alias ? p.Y : cv.take<int8_t>(size_t(L) * pl.Jx * pl.Kp);
    p.U = cv.take<uint8_t>(size_t(L) * pl.Jx * pl.Ip);
    p.stats_bytes = size_t(reinterpret_cast<char *>(p.ea) - reinterpret_cast<char *>(p.sa.amax));
    return p;
}

// Uploads the CRT tables to this translation unit's constant memory on the
// current device.
inline cudaError_t upload_tables() {
    static const CrtTables t = build_tables();
    return cudaMemcpyToSymbol(c_crt, &t, sizeof t);
}

}  // namespace
}  // namespace oz
}  // namespace bx
