// ozaki.cu -- scaling, slicing, modulus-count decision and CRT reconstruction
// of the emulated GEMM (see ozaki.h for the method), and its driver.
//
// Pipeline on one stream, with no host synchronisation:
//   stats(A), stats(B)  -> per-row max|x|, sum x^2, sum |x|, non-finite flag
//   decide              -> modulus count N (0 = native) and norm bound Q
//   slice(A), slice(B)  -> row exponents, int8 residues for l < N
//   residue GEMM        -> uint8 residues of every product (tcgen05)
//   reconstruct         -> exact CRT, unscale, alpha/beta epilogue
//   native guard        -> the native kernel runs only when N == 0
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "kernels.h"
#include "ozaki.h"
#include "profile.h"

namespace bx {
namespace oz {

const int kModuli[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                 223, 217, 211, 199, 197, 193, 191, 181, 179, 173};

namespace {

constexpr int kNumN = kMaxModuli - kMinModuli + 1;
constexpr int kP = 62;  // |scaled integer| < 2^62

struct CrtTables {
    uint32_t w[kNumN][kMaxModuli][kLimbs];  // CRT weights (M/m_l) * ((M/m_l)^-1 mod m_l)
    uint32_t M[kNumN][kLimbs];              // product of the first N moduli
    double Md[kNumN];                       // M as a double
    double invMd[kNumN];
    int Q[kNumN];                           // norm exponent bound: 2^(2Q) <= M/4
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
        }
    }
    return t;
}

// ---- device helpers ---------------------------------------------------------

template <typename T> struct Elem;
template <> struct Elem<double> { static constexpr bool cplx = false; };
template <> struct Elem<float> { static constexpr bool cplx = false; };
struct zpair { double re, im; };
template <> struct Elem<zpair> { static constexpr bool cplx = true; };

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
        const double *q = static_cast<const double *>(v.p) + 2 * off;
        re = q[0];
        im = v.conj ? -q[1] : q[1];
    } else {
        re = double(static_cast<const T *>(v.p)[off]);
        im = 0.0;
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr), __double_as_longlong(v));
}

// k-contiguous source: one warp per row, lanes stride over k.
template <typename T>
__global__ void stats_kc_kernel(View v, RowStats st) {
    const int64_t r = int64_t(blockIdx.x) * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
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

// row-contiguous source: one thread per row over a k-chunk, atomics combine.
template <typename T>
__global__ void stats_rc_kernel(View v, RowStats st, int64_t kchunk) {
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= v.R) return;
    const int64_t k0 = int64_t(blockIdx.y) * kchunk, k1 = min(v.K, k0 + kchunk);
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
__global__ void decide_kernel(RowStats sa, int64_t Ra, RowStats sb, int64_t Rb, int64_t K,
                              double unit, int mode, int forced, Decision *dec) {
    __shared__ double s_rho[2][32], s_h[2][32];
    __shared__ int s_bad[32];
    double rho[2] = {0, 0}, h[2] = {1e300, 1e300};
    int bad = 0;
    for (int side = 0; side < 2; ++side) {
        const RowStats &st = side ? sb : sa;
        const int64_t R = side ? Rb : Ra;
        for (int64_t r = threadIdx.x; r < R; r += blockDim.x) {
            bad |= st.flags[r];
            const double n1 = st.sumabs[r];
            if (n1 > 0) {
                const double n2 = sqrt(st.sumsq[r]);
                rho[side] = fmax(rho[side], n2 * sqrt(double(K)) / n1);
                h[side] = fmin(h[side], log2(n2 / st.amax[r]));
            }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
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
    if (threadIdx.x != 0) return;
    const int nw = blockDim.x / 32;
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

__device__ __forceinline__ uint32_t modulus_of(int l) {
    switch (l) {
        case 0: return 256; case 1: return 255; case 2: return 253; case 3: return 251;
        case 4: return 247; case 5: return 241; case 6: return 239; case 7: return 233;
        case 8: return 229; case 9: return 227; case 10: return 223; case 11: return 217;
        case 12: return 211; case 13: return 199; case 14: return 197; case 15: return 193;
        case 16: return 191; case 17: return 181; case 18: return 179; default: return 173;
    }
}

// Symmetric residue of a (|v| < 2^63) modulo the l-th modulus, as int8. With
// l a compile-time constant after unrolling, the divisions by m become
// multiply-high sequences.
__device__ __forceinline__ int32_t sym_residue(int64_t v, int l) {
    const uint32_t m = modulus_of(l);
    const uint32_t c32 = uint32_t((uint64_t(1) << 32) % m);
    const uint64_t a = v < 0 ? uint64_t(-v) : uint64_t(v);
    const uint32_t hi = uint32_t(a >> 32), lo = uint32_t(a);
    uint32_t r = ((hi % m) * c32 + (lo % m)) % m;
    if (v < 0 && r) r = m - r;
    int32_t s = int32_t(r);
    if (s > int32_t(m - 1) / 2) s -= int32_t(m);
    return s;
}

__device__ __forceinline__ int64_t scale_round(double x, int e) {
    return __double2ll_rn(ldexp(x, e));
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

template <int ROLE>
__device__ __forceinline__ void put4(const SliceOut &o, int l, int64_t r, int64_t k,
                                     const int32_t (&re)[4], const int32_t (&im)[4]) {
    auto pack = [](int32_t a, int32_t b, int32_t c, int32_t d) {
        return (uint32_t(a) & 0xff) | ((uint32_t(b) & 0xff) << 8) | ((uint32_t(c) & 0xff) << 16) |
               ((uint32_t(d) & 0xff) << 24);
    };
    int8_t *base = o.p + int64_t(l) * o.plane;
    *reinterpret_cast<uint32_t *>(base + r * o.Kp + k) = pack(re[0], re[1], re[2], re[3]);
    if (ROLE == 1) {
        *reinterpret_cast<uint32_t *>(base + r * o.Kp + o.Kh + k) = pack(im[0], im[1], im[2], im[3]);
    } else if (ROLE == 2) {
        *reinterpret_cast<uint32_t *>(base + r * o.Kp + o.Kh + k) =
            pack(-im[0], -im[1], -im[2], -im[3]);
        *reinterpret_cast<uint32_t *>(base + (o.Rp + r) * o.Kp + k) =
            pack(im[0], im[1], im[2], im[3]);
        *reinterpret_cast<uint32_t *>(base + (o.Rp + r) * o.Kp + o.Kh + k) =
            pack(re[0], re[1], re[2], re[3]);
    }
}

// k-contiguous source: a thread scales 4 consecutive k of one row and writes
// their residues for every modulus as one 4-byte word per plane.
// grid (Kc/64, Rp/16), block 256 = 16 (k groups of 4) x 16 rows.
template <typename T, int ROLE>
__global__ void slice_kc_kernel(View v, RowStats st, const Decision *dec, int *expo, SliceOut o) {
    const int nmod = dec->nmod;
    if (nmod == 0) return;
    const int Q = dec->q;
    const int64_t r = int64_t(blockIdx.y) * 16 + (threadIdx.x >> 4);
    const int64_t k = int64_t(blockIdx.x) * 64 + (threadIdx.x & 15) * 4;
    int e = 0;
    if (r < v.R) e = row_exponent(st.amax[r], st.sumsq[r], Q, v.K);
    if (blockIdx.x == 0 && (threadIdx.x & 15) == 0 && r < v.R) expo[r] = e;
    int64_t vr[4], vi[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double re = 0, im = 0;
        if (r < v.R && k + q < v.K) load_elem<T>(v, r, k + q, true, re, im);
        vr[q] = scale_round(re, e);
        vi[q] = scale_round(im, e);
    }
#pragma unroll
    for (int l = 0; l < kMaxModuli; ++l) {
        if (l < nmod) {
            int32_t rr[4], ri[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                rr[q] = sym_residue(vr[q], l);
                ri[q] = ROLE ? sym_residue(vi[q], l) : 0;
            }
            put4<ROLE>(o, l, r, k, rr, ri);
        }
    }
}

// row-contiguous source: a 64 (rows) x 64 (k) tile is read along rows,
// scaled, and its residues are transposed through shared memory so that the
// k-contiguous output rows are written with 4-byte words.
template <typename T, int ROLE>
__global__ void slice_rc_kernel(View v, RowStats st, const Decision *dec, int *expo, SliceOut o) {
    const int nmod = dec->nmod;
    if (nmod == 0) return;
    const int Q = dec->q;
    constexpr int CPL = ROLE ? 2 : 1;  // components
    __shared__ int8_t tile[CPL][64][64 + 4];
    __shared__ int s_e[64];
    const int64_t r0 = int64_t(blockIdx.y) * 64, k0 = int64_t(blockIdx.x) * 64;
    const int tr = threadIdx.x & 63, tk = threadIdx.x >> 6;  // tk in 0..3
    const int64_t r = r0 + tr;
    if (tk == 0) {
        int e = 0;
        if (r < v.R) e = row_exponent(st.amax[r], st.sumsq[r], Q, v.K);
        s_e[tr] = e;
        if (blockIdx.x == 0 && r < v.R) expo[r] = e;
    }
    __syncthreads();
    const int e = s_e[tr];
    int64_t vr[16], vi[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int64_t k = k0 + tk + 4 * i;
        double re = 0, im = 0;
        if (r < v.R && k < v.K) load_elem<T>(v, r, k, false, re, im);
        vr[i] = scale_round(re, e);
        vi[i] = scale_round(im, e);
    }
    // writer mapping: thread -> (row wr, 4 consecutive k at wk)
    const int wr = threadIdx.x >> 2, wk = (threadIdx.x & 3) * 16;
#pragma unroll
    for (int l = 0; l < kMaxModuli; ++l) {
        if (l < nmod) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                tile[0][tk + 4 * i][tr] = int8_t(sym_residue(vr[i], l));
                if (ROLE) tile[CPL - 1][tk + 4 * i][tr] = int8_t(sym_residue(vi[i], l));
            }
            __syncthreads();
            // thread writes 16 k of row (r0 + wr): 4 words per component
#pragma unroll
            for (int q = 0; q < 16; q += 4) {
                int32_t re4[4], im4[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    re4[u] = tile[0][wk + q + u][wr];
                    im4[u] = ROLE ? tile[CPL - 1][wk + q + u][wr] : 0;
                }
                put4<ROLE>(o, l, r0 + wr, k0 + wk + q, re4, im4);
            }
            __syncthreads();
        }
    }
}

// ---- reconstruction -----------------------------------------------------------

// CRT value of the residues u[0..n) for modulus count n, as a double
// (correctly rounded from the exact symmetric integer).
__device__ double crt_to_double(const uint32_t *u, int n) {
    const int ni = n - kMinModuli;
    uint64_t acc[kLimbs];
#pragma unroll
    for (int t = 0; t < kLimbs; ++t) acc[t] = 0;
    for (int l = 0; l < n; ++l) {
        const uint32_t ul = u[l];
#pragma unroll
        for (int t = 0; t < kLimbs; ++t) acc[t] += uint64_t(ul) * c_crt.w[ni][l][t];
    }
    // normalise to 32-bit limbs (S < 2^13 M < 2^192)
    uint32_t s[kLimbs];
    uint64_t carry = 0;
#pragma unroll
    for (int t = 0; t < kLimbs; ++t) {
        const uint64_t v = acc[t] + carry;
        s[t] = uint32_t(v);
        carry = v >> 32;
    }
    // q = floor(S / M), estimated in double and corrected below
    double sd = 0;
#pragma unroll
    for (int t = kLimbs - 1; t >= 0; --t) sd = sd * 4294967296.0 + double(s[t]);
    sd += double(carry) * 6277101735386680763835789423207666416102355444464034512896.0;  // 2^192
    int64_t q = int64_t(floor(sd * c_crt.invMd[ni]));
    if (q < 0) q = 0;
    // X = S - q M (may be negative by < M, or >= M by < M)
    int64_t borrow = 0;
    uint32_t x[kLimbs];
    {
        uint64_t qc = 0;
#pragma unroll
        for (int t = 0; t < kLimbs; ++t) {
            const uint64_t qm = uint64_t(q) * c_crt.M[ni][t] + qc;
            qc = qm >> 32;
            const int64_t d = int64_t(s[t]) - int64_t(uint32_t(qm)) - borrow;
            x[t] = uint32_t(d);
            borrow = d < 0 ? 1 : 0;
        }
        borrow = borrow + int64_t(qc) - int64_t(carry);  // > 0: X negative
    }
    auto add_m = [&](int sign) {  // x += sign * M
        int64_t c = 0;
#pragma unroll
        for (int t = 0; t < kLimbs; ++t) {
            const int64_t d = int64_t(x[t]) + sign * int64_t(c_crt.M[ni][t]) + c;
            x[t] = uint32_t(d);
            c = d >> 32;
        }
        return c;
    };
    if (borrow > 0) add_m(1);  // X < 0
    // X >= M ?
    bool ge = true;
#pragma unroll
    for (int t = kLimbs - 1; t >= 0; --t) {
        if (x[t] != c_crt.M[ni][t]) {
            ge = x[t] > c_crt.M[ni][t];
            break;
        }
    }
    if (ge) add_m(-1);
    // symmetric: X >= M/2 -> X - M (use 2X >= M)
    bool neg = false;
    {
        uint32_t x2[kLimbs];
        uint32_t c = 0;
#pragma unroll
        for (int t = 0; t < kLimbs; ++t) {
            x2[t] = (x[t] << 1) | c;
            c = x[t] >> 31;
        }
        bool gem = true;
#pragma unroll
        for (int t = kLimbs - 1; t >= 0; --t) {
            if (x2[t] != c_crt.M[ni][t]) {
                gem = x2[t] > c_crt.M[ni][t];
                break;
            }
        }
        if (gem) {
            // |X - M| = M - X
            int64_t b = 0;
#pragma unroll
            for (int t = 0; t < kLimbs; ++t) {
                const int64_t d = int64_t(c_crt.M[ni][t]) - int64_t(x[t]) - b;
                x[t] = uint32_t(d);
                b = d < 0 ? 1 : 0;
            }
            neg = true;
        }
    }
    // magnitude -> double, correctly rounded: a 64-bit window whose bit 63 is
    // the leading one, every lower bit folded into a sticky bit 0 (bit 0 lies
    // below the 53-bit rounding point, so round-to-nearest-even stays exact)
    int top = -1;
#pragma unroll
    for (int t = kLimbs - 1; t >= 0; --t)
        if (top < 0 && x[t]) top = t;
    if (top < 0) return 0.0;
    const uint64_t hi64 = (uint64_t(x[top]) << 32) | (top >= 1 ? x[top - 1] : 0u);
    const uint32_t lo32 = top >= 2 ? x[top - 2] : 0u;
    uint32_t sticky = 0;
    for (int t = top - 3; t >= 0; --t) sticky |= x[t];
    const int lz = __clzll(hi64);  // < 32 because x[top] != 0
    uint64_t win = hi64 << lz;
    if (lz) {
        win |= uint64_t(lo32) >> (32 - lz);
        sticky |= lo32 << lz;
    } else {
        sticky |= lo32;
    }
    if (sticky) win |= 1;
    const double d = ldexp(__ull2double_rn(win), 32 * (top - 1) - lz);
    return neg ? -d : d;
}

template <typename T> struct OutT;
template <> struct OutT<double> { using type = double; };
template <> struct OutT<float> { using type = float; };

// Real outputs: thread -> 4 consecutive rows i of one column j.
template <typename T>
__global__ void reconstruct_real_kernel(const uint8_t *U, int64_t Jp, int64_t Ip, int64_t M,
                                        int64_t N, const int *ea, const int *fb, const Decision *dec,
                                        double alpha, double beta, int beta_zero, T *C,
                                        int64_t ldc) {
    const int n = dec->nmod;
    if (n == 0) return;
    const int64_t j = blockIdx.y;
    const int64_t i0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * 4;
    if (i0 >= M || j >= N) return;
    uint32_t u[4][kMaxModuli];
    for (int l = 0; l < n; ++l) {
        const uchar4 w = *reinterpret_cast<const uchar4 *>(U + int64_t(l) * Jp * Ip + j * Ip + i0);
        u[0][l] = w.x; u[1][l] = w.y; u[2][l] = w.z; u[3][l] = w.w;
    }
    const int fj = fb[j];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int64_t i = i0 + q;
        if (i >= M) break;
        const double val = ldexp(crt_to_double(u[q], n), -(ea[i] + fj));
        T *cp = C + i + j * ldc;
        double r = alpha * val;
        if (!beta_zero) r = fma(beta, double(*cp), r);
        *cp = T(r);
    }
}

// Complex outputs: the residue block of Re(C) is rows [0, Jp) of U, Im(C)
// rows [Jp, 2Jp).
__global__ void reconstruct_cplx_kernel(const uint8_t *U, int64_t Jp, int64_t Ip, int64_t M,
                                        int64_t N, const int *ea, const int *fb,
                                        const Decision *dec, double ar, double ai, double br,
                                        double bi, int beta_zero, double *C, int64_t ldc) {
    const int n = dec->nmod;
    if (n == 0) return;
    const int64_t j = blockIdx.y;
    const int64_t i0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) * 4;
    if (i0 >= M || j >= N) return;
    const int64_t plane = 2 * Jp * Ip;
    const int fj = fb[j];
    uint32_t ur[4][kMaxModuli], ui[4][kMaxModuli];
    for (int l = 0; l < n; ++l) {
        const uchar4 a = *reinterpret_cast<const uchar4 *>(U + int64_t(l) * plane + j * Ip + i0);
        const uchar4 b =
            *reinterpret_cast<const uchar4 *>(U + int64_t(l) * plane + (Jp + j) * Ip + i0);
        ur[0][l] = a.x; ur[1][l] = a.y; ur[2][l] = a.z; ur[3][l] = a.w;
        ui[0][l] = b.x; ui[1][l] = b.y; ui[2][l] = b.z; ui[3][l] = b.w;
    }
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        const int64_t i = i0 + q;
        if (i >= M) break;
        const int sc = -(ea[i] + fj);
        const double xr = ldexp(crt_to_double(ur[q], n), sc);
        const double xi = ldexp(crt_to_double(ui[q], n), sc);
        double *cp = C + 2 * (i + j * ldc);
        double vr = ar * xr - ai * xi, vi = ar * xi + ai * xr;
        if (!beta_zero) {
            const double cr = cp[0], ci = cp[1];
            vr += br * cr - bi * ci;
            vi += br * ci + bi * cr;
        }
        cp[0] = vr;
        cp[1] = vi;
    }
}

std::once_flag g_tables_once;
int g_tables_status = BLASX_OK;

}  // namespace

int upload_crt_tables() {
    std::call_once(g_tables_once, [] {
        static CrtTables t = build_tables();
        if (cudaMemcpyToSymbol(c_crt, &t, sizeof t) != cudaSuccess) g_tables_status = BLASX_ERR_CUDA;
    });
    if (g_tables_status != BLASX_OK) return set_error(g_tables_status, "CRT table upload failed");
    return BLASX_OK;
}

int prepare_crt_tables_current_device() {
    static const CrtTables t = build_tables();
    BX_CUDA(cudaMemcpyToSymbol(c_crt, &t, sizeof t));
    return BLASX_OK;
}

}  // namespace oz

// --------------------------------------------------------------------------
// driver
// --------------------------------------------------------------------------

namespace {

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

template <typename T>
int launch_stats(const oz::View &v, bool kc, const oz::RowStats &st, cudaStream_t s) {
    if (v.R == 0) return BLASX_OK;
    if (kc) {
        oz::stats_kc_kernel<T><<<unsigned((v.R + 7) / 8), 256, 0, s>>>(v, st);
    } else {
        const int64_t kchunk = 512;
        dim3 grid(unsigned((v.R + 255) / 256), unsigned((v.K + kchunk - 1) / kchunk));
        oz::stats_rc_kernel<T><<<grid, 256, 0, s>>>(v, st, kchunk);
    }
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

template <typename T, int ROLE>
int launch_slice(const oz::View &v, bool kc, const oz::RowStats &st, const oz::Decision *dec,
                 int *expo, const oz::SliceOut &o, int64_t Kc, cudaStream_t s) {
    if (kc) {
        dim3 grid(unsigned(Kc / 64), unsigned(o.Rp / 16));
        oz::slice_kc_kernel<T, ROLE><<<grid, 256, 0, s>>>(v, st, dec, expo, o);
    } else {
        dim3 grid(unsigned(Kc / 64), unsigned(o.Rp / 64));
        oz::slice_rc_kernel<T, ROLE><<<grid, 256, 0, s>>>(v, st, dec, expo, o);
    }
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

int forced_moduli() {
    static const int f = [] {
        const char *e = getenv("BLASX_OZAKI_MODULI");
        const int v = e ? atoi(e) : 0;
        return (v >= oz::kMinModuli && v <= oz::kMaxModuli) ? v : 0;
    }();
    return f;
}

// Padded extents and scratch size of one emulated GEMM.
struct Plan {
    int64_t M, N, K, Kh, Kp, Kc, Ip, Jp, Jx;
    size_t bytes;
};

Plan make_plan(const Gemm &g) {
    const bool cplx = g.dt == DType::C128;
    const int64_t L = oz::kMaxModuli;
    Plan p;
    p.M = g.M; p.N = g.N; p.K = g.K;
    p.Kh = cplx ? oz::pad(p.K, 64) : 0;
    p.Kp = cplx ? 2 * p.Kh : oz::pad(p.K, oz::kTileK);
    p.Kc = cplx ? p.Kh : p.Kp;  // k extent covered by the slice kernels
    p.Ip = oz::pad(p.M, oz::kTileI);
    p.Jp = oz::pad(p.N, oz::kTileJ);
    p.Jx = cplx ? 2 * p.Jp : p.Jp;  // X rows (Re block + Im block)
    p.bytes = 256 * 16 + (3 * sizeof(double) + 2 * sizeof(int)) * size_t(p.M + p.N) +
              sizeof(oz::Decision) + sizeof(int) + size_t(L) * p.Ip * p.Kp +
              size_t(L) * p.Jx * p.Kp + size_t(L) * p.Jx * p.Ip;
    return p;
}

// The whole emulated pipeline on a caller-provided workspace of
// make_plan(g).bytes bytes: no allocation. The device decision and error
// flag are copied to the given host slots when they are not null.
template <typename T>
int ozaki_run(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms, void *dec_host,
              int *err_host) {
    constexpr bool CPLX = oz::Elem<T>::cplx;
    const Plan pl = make_plan(g);
    const int64_t M = pl.M, N = pl.N, K = pl.K, Kh = pl.Kh, Kp = pl.Kp, Kc = pl.Kc;
    const int64_t Ip = pl.Ip, Jp = pl.Jp, Jx = pl.Jx;
    const int64_t L = oz::kMaxModuli;
    Carve cv{static_cast<char *>(ws)};
    oz::RowStats sa{cv.take<double>(M), cv.take<double>(M), cv.take<double>(M), cv.take<int>(M)};
    oz::RowStats sb{cv.take<double>(N), cv.take<double>(N), cv.take<double>(N), cv.take<int>(N)};
    int *ea = cv.take<int>(M), *fb = cv.take<int>(N);
    oz::Decision *dec = cv.take<oz::Decision>(1);
    int *err = cv.take<int>(1);
    int8_t *Y = cv.take<int8_t>(size_t(L) * Ip * Kp);
    int8_t *X = cv.take<int8_t>(size_t(L) * Jx * Kp);
    uint8_t *U = cv.take<uint8_t>(size_t(L) * Jx * Ip);
    const size_t stats_bytes = reinterpret_cast<char *>(ea) - static_cast<char *>(ws);
    cudaEvent_t ev0 = prof::mark(s);
    BX_CUDA(cudaMemsetAsync(ws, 0, stats_bytes, s));
    BX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));

    // op(A) rows i over k; op(B) columns j over k
    oz::View va{g.A, g.lda, M, K, g.ta == ConjT};
    oz::View vb{g.B, g.ldb, N, K, g.tb == ConjT};
    const bool akc = g.ta != NoTrans, bkc = g.tb == NoTrans;
    BX_TRY(launch_stats<T>(va, akc, sa, s));
    BX_TRY(launch_stats<T>(vb, bkc, sb, s));
    const double unit = std::is_same<T, float>::value ? std::ldexp(1.0, -24) : std::ldexp(1.0, -53);
    oz::decide_kernel<<<1, 1024, 0, s>>>(sa, M, sb, N, K, unit, mode, forced_moduli(), dec);
    BX_CUDA(cudaGetLastError());
    count_launch();

    oz::SliceOut oy{Y, Ip, Kp, Kh, Ip * Kp};
    oz::SliceOut ox{X, Jp, Kp, Kh, Jx * Kp};
    if (CPLX) {
        BX_TRY((launch_slice<T, 1>(va, akc, sa, dec, ea, oy, Kc, s)));
        BX_TRY((launch_slice<T, 2>(vb, bkc, sb, dec, fb, ox, Kc, s)));
    } else {
        BX_TRY((launch_slice<T, 0>(va, akc, sa, dec, ea, oy, Kc, s)));
        BX_TRY((launch_slice<T, 0>(vb, bkc, sb, dec, fb, ox, Kc, s)));
    }
    cudaEvent_t ev1 = prof::mark(s);
    BX_TRY(oz::launch_residue_gemm(X, Y, U, Jx, Ip, Kp, dec, err, num_sms, s));
    cudaEvent_t ev2 = prof::mark(s);

    dim3 rgrid(unsigned((M + 4 * 128 - 1) / (4 * 128)), unsigned(N));
    if constexpr (CPLX) {
        oz::reconstruct_cplx_kernel<<<rgrid, 128, 0, s>>>(U, Jp, Ip, M, N, ea, fb, dec, g.alpha.re,
                                                          g.alpha.im, g.beta.re, g.beta.im,
                                                          g.beta_zero() ? 1 : 0,
                                                          static_cast<double *>(g.C), g.ldc);
    } else {
        oz::reconstruct_real_kernel<T><<<rgrid, 128, 0, s>>>(
            U, Jx, Ip, M, N, ea, fb, dec, g.alpha.re, g.beta.re, g.beta_zero() ? 1 : 0,
            static_cast<T *>(g.C), g.ldc);
    }
    BX_CUDA(cudaGetLastError());
    count_launch();

    cudaEvent_t ev3 = prof::mark(s);

    // native fallback, decided on the device (runs only when nmod == 0)
    Gemm gn = g;
    gn.guard = &dec->nmod;
    if (g.dt == DType::F32) BX_TRY(launch_gemm_simt(gn, s));
    else BX_TRY(launch_gemm_dmma(gn, s));
    cudaEvent_t ev4 = prof::mark(s);
    prof::span(prof::kSlice, ev0, ev1);
    prof::span(prof::kResidueGemm, ev1, ev2);
    prof::span(prof::kReconstruct, ev2, ev3);
    prof::span(prof::kNative, ev3, ev4);

    // record the decision for blasx_get_call_stats (lands when the stream does)
    if (dec_host)
        BX_CUDA(cudaMemcpyAsync(dec_host, dec, sizeof(oz::Decision), cudaMemcpyDeviceToHost, s));
    if (err_host) BX_CUDA(cudaMemcpyAsync(err_host, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    call_stats().path = 2;
    return BLASX_OK;
}

template <typename T> int ozaki_t(const Gemm &g, cudaStream_t s, int mode) {
    Context *ctx = context();
    if (!ctx) return last_status();
    BX_TRY(oz::upload_crt_tables());
    const Plan pl = make_plan(g);
    void *ws = nullptr;
    BX_CUDA(cudaMallocAsync(&ws, pl.bytes, s));
    struct Free {
        void *p;
        cudaStream_t s;
        ~Free() { cudaFreeAsync(p, s); }
    } free_ws{ws, s};
    return ozaki_run<T>(g, s, mode, ws, ctx->num_sms, ctx->last_decision, ctx->last_error_flag);
}

}  // namespace

int ozaki_gemm(const Gemm &g, cudaStream_t s, int mode) {
    switch (g.dt) {
        case DType::F64: return ozaki_t<double>(g, s, mode);
        case DType::F32: return ozaki_t<float>(g, s, mode);
        default: return ozaki_t<oz::zpair>(g, s, mode);
    }
}

size_t ozaki_scratch_bytes(const Gemm &g) { return make_plan(g).bytes; }

int ozaki_gemm_in(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms) {
    switch (g.dt) {
        case DType::F64: return ozaki_run<double>(g, s, mode, ws, num_sms, nullptr, nullptr);
        case DType::F32: return ozaki_run<float>(g, s, mode, ws, num_sms, nullptr, nullptr);
        default: return ozaki_run<oz::zpair>(g, s, mode, ws, num_sms, nullptr, nullptr);
    }
}

}  // namespace bx
