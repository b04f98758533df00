// trsm.cu -- triangular solve (cblas_?trsm) and triangular multiply
// (cblas_?trmm) with many right-hand sides on device operands.
//
// op(A) X = alpha B (left) or X op(A) = alpha B (right) is solved by
// recursive halving of the order-K triangle: solve the first half, update
// the second half's right-hand sides with one GEMM (device_gemm: native, or
// emulated on the INT8 tensor cores where the precision mode selects it),
// solve the second half. The top-level updates carry most of the K^2 * (M or
// N) work with K up to K/2, the shape the emulated GEMM needs; blocks of at
// most 64 rows (32 complex) are solved by substitution in one kernel.
//
// Every GEMM reads op(A) only in an off-diagonal rectangle inside the stored
// triangle, and the substitution kernel reads only the stored triangle of its
// diagonal block (not the diagonal when it is unit): the other triangle of A
// is never read.
#include <algorithm>

#include "arith.cuh"
#include "kernels.h"

namespace bx {
namespace {

// Order of a substitution block: one right-hand-side vector of it lives in
// one thread's registers (64 doubles, or 32 complex doubles).
template <typename T> struct LeafDim {
    static constexpr int n = 64;
};
template <> struct LeafDim<z2> {
    static constexpr int n = 32;
};
template <> struct LeafDim<c2> {
    static constexpr int n = 32;
};
constexpr int kLeafVecs = 64;     // right-hand-side vectors per CTA
constexpr int kLanes = 4;         // lanes per vector: lane j owns rows j, j + 4, ...
constexpr int kLeafThreads = kLeafVecs * kLanes;

int leaf_order(DType dt) { return is_complex(dt) ? 32 : 64; }

template <typename T> __device__ inline T negate(T a) { return -a; }
template <> __device__ inline z2 negate<z2>(z2 a) { return {-a.re, -a.im}; }
template <> __device__ inline c2 negate<c2>(c2 a) { return {-a.re, -a.im}; }

template <typename T> __device__ inline T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <> __device__ inline z2 shfl<z2>(z2 v, int src) {
    return {__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}
template <> __device__ inline c2 shfl<c2>(c2 v, int src) {
    return {__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}

// Solves S x = c for nvec vectors at once, S the bs x bs (bs <= L) system
// matrix of one diagonal block: S = op(A_block) for a left solve, the
// transpose of op(A_block) for a right solve (x op(A) = c is op(A)^T x^T =
// c^T). S[i][k] is A[i + k lda] (s_trans = 0) or A[k + i lda] (s_trans = 1),
// conjugated when s_conj. S is lower (FORWARD substitution) or upper; only
// that triangle of S, and its diagonal unless UNIT, is read. Vector v,
// element i: left: C[i + v ldc] (columns of B); right: C[v + i ldc] (rows of
// B). Each vector is scaled by `scale` (alpha) on load.
//
// Shared memory holds S by columns (St[k * L + i] = S[i][k]), zero outside
// the triangle, the reciprocals of its diagonal and, for a left solve, the
// CTA's vectors: they are columns of B, which consecutive threads load and
// store row by row (coalesced) through shared memory. Four adjacent lanes
// solve one vector held in their registers, lane j owning rows j, j + 4, ...
// The substitution is unrolled over the L x L block, so every register index
// is a compile-time constant; at step k the lane owning row k scales it by
// 1 / S[k][k], a shuffle hands x_k to the other three, and each lane updates
// its later rows (no barrier). A block smaller than L is padded with zero
// right-hand sides and unit diagonal, which leave the real rows unchanged.
template <typename T, bool FORWARD, bool UNIT>
__global__ void __launch_bounds__(kLeafThreads)
    trsm_leaf_kernel(const T *__restrict__ A, int64_t lda, T *__restrict__ C, int64_t ldc, int bs,
                     int64_t nvec, int left, int s_trans, int s_conj, T scale) {
    using Ar = Arith<T>;
    constexpr int L = LeafDim<T>::n;
    constexpr int R = L / kLanes;  // rows per lane
    extern __shared__ __align__(16) unsigned char smem[];
    T *St = reinterpret_cast<T *>(smem);  // St[k * L + i] = S[i][k]
    T *rdiag = St + L * L;                // 1 / S[k][k]
    T *Cs = rdiag + L;                    // left: Cs[v * (L + 1) + i], this CTA's vectors
    const int64_t v0 = int64_t(blockIdx.x) * kLeafVecs;
    const int tid = threadIdx.x;
    // global -> shared: every load of a thread is issued before its stores
    constexpr int kStPer = L * L / kLeafThreads, kCsPer = L * kLeafVecs / kLeafThreads;
    static_assert(kStPer * kLeafThreads == L * L && kCsPer * kLeafThreads == L * kLeafVecs, "whole batches");
    if (left) {  // a left vector is a column of B: consecutive threads take consecutive rows
        T tmp[kCsPer];
#pragma unroll
        for (int q = 0; q < kCsPer; ++q) {
            const int e = tid + q * kLeafThreads, i = e % L, vv = e / L;
            tmp[q] = (i < bs && v0 + vv < nvec) ? C[i + (v0 + vv) * ldc] : Ar::zero();
        }
#pragma unroll
        for (int q = 0; q < kCsPer; ++q) {
            const int e = tid + q * kLeafThreads;
            Cs[(e / L) * (L + 1) + e % L] = tmp[q];
        }
    }
    {
        T tmp[kStPer];
#pragma unroll
        for (int q = 0; q < kStPer; ++q) {
            const int e = tid + q * kLeafThreads, i = e % L, k = e / L;
            tmp[q] = Ar::zero();
            if (i < bs && k < bs && (FORWARD ? i > k : i < k))
                tmp[q] = s_trans ? A[k + int64_t(i) * lda] : A[i + int64_t(k) * lda];
        }
#pragma unroll
        for (int q = 0; q < kStPer; ++q) St[tid + q * kLeafThreads] = s_conj ? Ar::conj(tmp[q]) : tmp[q];
    }
    if (tid < L) {
        T r = Ar::one();
        if (!UNIT && tid < bs) {
            T d = A[tid + int64_t(tid) * lda];
            if (s_conj) d = Ar::conj(d);
            r = quot(Ar::one(), d);
        }
        rdiag[tid] = r;
    }
    __syncthreads();
    const int j = tid % kLanes, vl = tid / kLanes;
    const int64_t v = v0 + vl;
    const bool live = v < nvec;
    const int base = tid & ~(kLanes - 1);  // lane 0 of this vector's group
    T c[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        const int i = j + kLanes * m;
        c[m] = Ar::zero();
        if (i < bs && live) c[m] = Ar::mul(scale, left ? Cs[vl * (L + 1) + i] : C[v + int64_t(i) * ldc]);
    }
#pragma unroll
    for (int s = 0; s < L; ++s) {
        const int k = FORWARD ? s : L - 1 - s;
        const int mk = k / kLanes, jk = k % kLanes;
        if (!UNIT && j == jk) c[mk] = Ar::mul(c[mk], rdiag[k]);
        const T xk = shfl(c[mk], base + jk);
        const T *col = St + k * L;
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const int i = j + kLanes * m;
            if (FORWARD ? (kLanes * m + kLanes - 1 > k && i > k) : (kLanes * m < k && i < k))
                c[m] = Ar::fma(negate(col[i]), xk, c[m]);
        }
    }
    if (!left) {
        if (live)
#pragma unroll
            for (int m = 0; m < R; ++m) {
                const int i = j + kLanes * m;
                if (i < bs) C[v + int64_t(i) * ldc] = c[m];
            }
        return;
    }
#pragma unroll
    for (int m = 0; m < R; ++m) Cs[vl * (L + 1) + j + kLanes * m] = c[m];
    __syncthreads();
    for (int e = tid; e < L * kLeafVecs; e += kLeafThreads) {
        const int i = e % L, vv = e / L;
        if (i < bs && v0 + vv < nvec) C[i + (v0 + vv) * ldc] = Cs[vv * (L + 1) + i];
    }
}

template <typename T> size_t leaf_smem() {
    constexpr int L = LeafDim<T>::n;
    return sizeof(T) * (L * (L + 1) + kLeafVecs * (L + 1));
}

template <typename T, bool FORWARD, bool UNIT>
int launch_leaf_k(const Trsm &t, int64_t lo, int64_t hi, cplx scale, int s_trans, cudaStream_t s) {
    static const cudaError_t attr = cudaFuncSetAttribute(
        trsm_leaf_kernel<T, FORWARD, UNIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(leaf_smem<T>()));
    BX_CUDA(attr);
    const int64_t nvec = t.left ? t.N : t.M;
    const T *A = static_cast<const T *>(t.A) + lo + lo * t.lda;
    T *C = static_cast<T *>(t.B) + (t.left ? lo : lo * t.ldb);
    const int64_t blocks = (nvec + kLeafVecs - 1) / kLeafVecs;
    if (blocks > 0x7fffffff) return set_error(BLASX_ERR_UNSUPPORTED, "trsm: too many right-hand sides");
    const bool conj = is_complex(t.dt) && t.trans == ConjT;
    trsm_leaf_kernel<T, FORWARD, UNIT><<<unsigned(blocks), kLeafThreads, leaf_smem<T>(), s>>>(
        A, t.lda, C, t.ldb, int(hi - lo), nvec, t.left, s_trans, conj, from_cplx<T>(scale));
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

template <typename T>
int launch_leaf_t(const Trsm &t, int64_t lo, int64_t hi, cplx scale, int s_trans, int forward, cudaStream_t s) {
    if (forward)
        return t.unit ? launch_leaf_k<T, true, true>(t, lo, hi, scale, s_trans, s)
                      : launch_leaf_k<T, true, false>(t, lo, hi, scale, s_trans, s);
    return t.unit ? launch_leaf_k<T, false, true>(t, lo, hi, scale, s_trans, s)
                  : launch_leaf_k<T, false, false>(t, lo, hi, scale, s_trans, s);
}

int launch_leaf(const Trsm &t, int64_t lo, int64_t hi, cplx scale, int s_trans, int forward, cudaStream_t s) {
    switch (t.dt) {
        case DType::F32: return launch_leaf_t<float>(t, lo, hi, scale, s_trans, forward, s);
        case DType::F64: return launch_leaf_t<double>(t, lo, hi, scale, s_trans, forward, s);
        case DType::C64: return launch_leaf_t<c2>(t, lo, hi, scale, s_trans, forward, s);
        default: return launch_leaf_t<z2>(t, lo, hi, scale, s_trans, forward, s);
    }
}

struct Range {
    int64_t lo, hi;
    int64_t size() const { return hi - lo; }
};

// The system matrix S of the blocks (see trsm_leaf_kernel) is A or A^T:
// s_trans = 1 when S = A^T. Substitution runs forward when S is lower.
int s_trans_of(const Trsm &t) { return t.left ? t.trans != NoTrans : t.trans == NoTrans; }
bool forward_of(const Trsm &t) { return t.lower != bool(s_trans_of(t)); }

// The two halves of [lo, hi) in solve order: the first has a multiple of
// the leaf order rows.
void split(const Trsm &t, Range r, Range *first, Range *second) {
    const int64_t n = r.size(), lf = leaf_order(t.dt);
    const int64_t half = std::min(n - 1, (n / 2 + lf - 1) / lf * lf);
    if (forward_of(t)) {
        *first = {r.lo, r.lo + half};
        *second = {r.lo + half, r.hi};
    } else {
        *first = {r.hi - half, r.hi};
        *second = {r.lo, r.hi - half};
    }
}

// B[tgt] = beta B[tgt] + alpha op(A)[tgt, src] B[src] (left) or
// B[:, tgt] = beta B[:, tgt] + alpha B[:, src] op(A)[src, tgt] (right).
Gemm update_gemm(const Trsm &t, Range tgt, Range src, cplx alpha, cplx beta) {
    const size_t es = elem_size(t.dt);
    const char *A = static_cast<const char *>(t.A);
    char *B = static_cast<char *>(t.B);
    const int tr = (t.trans == ConjT && !is_complex(t.dt)) ? TransT : t.trans;
    Gemm g;
    g.dt = t.dt;
    g.alpha = alpha;
    g.beta = beta;
    g.K = src.size();
    if (t.left) {
        g.M = tgt.size();
        g.N = t.N;
        g.ta = tr;
        g.A = tr == NoTrans ? A + (tgt.lo + src.lo * t.lda) * es : A + (src.lo + tgt.lo * t.lda) * es;
        g.lda = t.lda;
        g.tb = NoTrans;
        g.B = B + src.lo * es;
        g.ldb = t.ldb;
        g.C = B + tgt.lo * es;
    } else {
        g.M = t.M;
        g.N = tgt.size();
        g.ta = NoTrans;
        g.A = B + src.lo * t.ldb * es;
        g.lda = t.ldb;
        g.tb = tr;
        g.B = tr == NoTrans ? A + (src.lo + tgt.lo * t.lda) * es : A + (tgt.lo + src.lo * t.lda) * es;
        g.ldb = t.lda;
        g.C = B + tgt.lo * t.ldb * es;
    }
    g.ldc = t.ldb;
    return g;
}

constexpr cplx kMinusOne{-1.0, 0.0}, kOne{1.0, 0.0};

int solve(const Trsm &t, Range r, cplx scale, cudaStream_t s, bool *emulated) {
    if (r.size() <= leaf_order(t.dt)) return launch_leaf(t, r.lo, r.hi, scale, s_trans_of(t), forward_of(t), s);
    Range first, second;
    split(t, r, &first, &second);
    BX_TRY(solve(t, first, scale, s, emulated));
    BX_TRY(device_gemm(update_gemm(t, second, first, kMinusOne, scale), s));
    if (call_stats().path == 2) *emulated = true;
    return solve(t, second, cplx{1.0, 0.0}, s, emulated);
}

// ---- TRMM: B = alpha op(A) B or alpha B op(A), in place -------------------
// With the vectors of B (columns for a left multiply, rows for a right one)
// the product is v <- alpha S v, S = op(A) or op(A)^T as for the solve. It
// recurses over halves P (earlier rows of S) and Q: for S lower,
// v_Q <- alpha S_QQ v_Q + alpha S_QP v_P needs the original v_P, so Q goes
// first (its multiply, then one GEMM update from P), then P; for S upper,
// P goes first. Every GEMM reads op(A) in an off-diagonal rectangle inside
// the stored triangle. A leaf of at most kTrmmLeaf rows multiplies by its
// diagonal block, completed (zeros, unit diagonal) in a scratch copy, on
// the native kernels: the emulated path never sees a triangle's tip, whose
// single nonzero per row would lose accuracy under per-row scaling.
constexpr int kTrmmLeaf = 256;

void trmm_split(const Trsm &t, Range r, Range *first, Range *second) {
    const int64_t n = r.size();
    const int64_t half = std::min(n - 1, (n / 2 + kTrmmLeaf - 1) / kTrmmLeaf * kTrmmLeaf);
    const Range lo{r.lo, r.lo + half}, hi{r.lo + half, r.hi};
    *first = forward_of(t) ? hi : lo;
    *second = forward_of(t) ? lo : hi;
}

int trmm_leaf(const Trsm &t, Range r, const TrmmScratch &w, cudaStream_t s) {
    const size_t es = elem_size(t.dt);
    const int64_t bs = r.size();
    const char *A = static_cast<const char *>(t.A);
    char *B = static_cast<char *>(t.B);
    BX_CUDA(cudaMemcpy2DAsync(w.diag, size_t(kTrmmLeaf) * es, A + (r.lo + r.lo * t.lda) * es, size_t(t.lda) * es,
                              size_t(bs) * es, size_t(bs), cudaMemcpyDeviceToDevice, s));
    const int form = t.lower ? (t.unit ? kTriLowerUnit : kTriLower) : (t.unit ? kTriUpperUnit : kTriUpper);
    BX_TRY(launch_complete_operand(t.dt, form, w.diag, kTrmmLeaf, bs, s));
    const int tr = (t.trans == ConjT && !is_complex(t.dt)) ? TransT : t.trans;
    Gemm g;
    g.dt = t.dt;
    g.alpha = t.alpha;
    g.beta = cplx{0.0, 0.0};
    g.K = bs;
    if (t.left) {  // rows r of B: B_r = alpha op(A_rr) B_r
        BX_CUDA(cudaMemcpy2DAsync(w.temp, size_t(w.ldt) * es, B + r.lo * es, size_t(t.ldb) * es, size_t(bs) * es,
                                  size_t(t.N), cudaMemcpyDeviceToDevice, s));
        g.M = bs; g.N = t.N;
        g.ta = tr; g.A = w.diag; g.lda = kTrmmLeaf;
        g.tb = NoTrans; g.B = w.temp; g.ldb = w.ldt;
        g.C = B + r.lo * es;
    } else {  // columns r of B: B_r = alpha B_r op(A_rr)
        BX_CUDA(cudaMemcpy2DAsync(w.temp, size_t(w.ldt) * es, B + r.lo * t.ldb * es, size_t(t.ldb) * es,
                                  size_t(t.M) * es, size_t(bs), cudaMemcpyDeviceToDevice, s));
        g.M = t.M; g.N = bs;
        g.ta = NoTrans; g.A = w.temp; g.lda = w.ldt;
        g.tb = tr; g.B = w.diag; g.ldb = kTrmmLeaf;
        g.C = B + r.lo * t.ldb * es;
    }
    g.ldc = t.ldb;
    return dmma_supported(g) ? launch_gemm_dmma(g, s) : launch_gemm_simt(g, s);
}

int multiply(const Trsm &t, Range r, const TrmmScratch &w, cudaStream_t s, bool *emulated) {
    if (r.size() <= kTrmmLeaf) return trmm_leaf(t, r, w, s);
    Range first, second;
    trmm_split(t, r, &first, &second);
    BX_TRY(multiply(t, first, w, s, emulated));
    BX_TRY(device_gemm(update_gemm(t, first, second, t.alpha, kOne), s));
    if (call_stats().path == 2) *emulated = true;
    return multiply(t, second, w, s, emulated);
}

// The same product out of place: part r of dst (B's layout) = alpha S_rr
// B_r, B unchanged. A leaf multiplies B's rows (or columns) by the completed
// diagonal block straight into dst, with no staging copy; every update
// reads B's original values, so the halves may go in either order.
int leaf_into(const Trsm &t, void *dst, Range r, const TrmmScratch &w, cudaStream_t s) {
    const size_t es = elem_size(t.dt);
    const int64_t bs = r.size();
    const char *A = static_cast<const char *>(t.A);
    const char *B = static_cast<const char *>(t.B);
    char *D = static_cast<char *>(dst);
    BX_CUDA(cudaMemcpy2DAsync(w.diag, size_t(kTrmmLeaf) * es, A + (r.lo + r.lo * t.lda) * es, size_t(t.lda) * es,
                              size_t(bs) * es, size_t(bs), cudaMemcpyDeviceToDevice, s));
    const int form = t.lower ? (t.unit ? kTriLowerUnit : kTriLower) : (t.unit ? kTriUpperUnit : kTriUpper);
    BX_TRY(launch_complete_operand(t.dt, form, w.diag, kTrmmLeaf, bs, s));
    const int tr = (t.trans == ConjT && !is_complex(t.dt)) ? TransT : t.trans;
    Gemm g;
    g.dt = t.dt;
    g.alpha = t.alpha;
    g.beta = cplx{0.0, 0.0};
    g.K = bs;
    if (t.left) {  // rows r: D_r = alpha op(A_rr) B_r
        g.M = bs; g.N = t.N;
        g.ta = tr; g.A = w.diag; g.lda = kTrmmLeaf;
        g.tb = NoTrans; g.B = B + r.lo * es; g.ldb = t.ldb;
        g.C = D + r.lo * es;
    } else {  // columns r: D_r = alpha B_r op(A_rr)
        g.M = t.M; g.N = bs;
        g.ta = NoTrans; g.A = B + r.lo * t.ldb * es; g.lda = t.ldb;
        g.tb = tr; g.B = w.diag; g.ldb = kTrmmLeaf;
        g.C = D + r.lo * t.ldb * es;
    }
    g.ldc = t.ldb;
    return dmma_supported(g) ? launch_gemm_dmma(g, s) : launch_gemm_simt(g, s);
}

int multiply_into(const Trsm &t, void *dst, Range r, const TrmmScratch &w, cudaStream_t s, bool *emulated) {
    if (r.size() <= kTrmmLeaf) return leaf_into(t, dst, r, w, s);
    Range first, second;
    trmm_split(t, r, &first, &second);
    BX_TRY(multiply_into(t, dst, first, w, s, emulated));
    Gemm g = update_gemm(t, first, second, t.alpha, kOne);
    g.C = static_cast<char *>(dst) + (static_cast<char *>(g.C) - static_cast<char *>(t.B));
    BX_TRY(device_gemm(g, s));
    if (call_stats().path == 2) *emulated = true;
    return multiply_into(t, dst, second, w, s, emulated);
}

}  // namespace

bool tri_forward(const Trsm &t) { return forward_of(t); }

Gemm tri_update_gemm(const Trsm &t, int64_t tgt_lo, int64_t tgt_hi, int64_t src_lo, int64_t src_hi) {
    return update_gemm(t, Range{tgt_lo, tgt_hi}, Range{src_lo, src_hi}, t.alpha, kOne);
}

int trsm_solve_part(const Trsm &t, int64_t lo, int64_t hi, cplx scale, cudaStream_t s, bool *emulated) {
    return solve(t, Range{lo, hi}, scale, s, emulated);
}

int trsm_update_part(const Trsm &t, int64_t tgt_lo, int64_t tgt_hi, int64_t src_lo, int64_t src_hi, cplx scale,
                     cudaStream_t s, bool *emulated) {
    BX_TRY(device_gemm(update_gemm(t, Range{tgt_lo, tgt_hi}, Range{src_lo, src_hi}, kMinusOne, scale), s));
    if (call_stats().path == 2) *emulated = true;
    return BLASX_OK;
}

Gemm trsm_top_update(const Trsm &t) {
    const Range all{0, t.order()};
    if (all.size() <= leaf_order(t.dt)) {
        Gemm g = update_gemm(t, all, all, kMinusOne, t.alpha);
        g.K = 0;
        return g;
    }
    Range first, second;
    split(t, all, &first, &second);
    return update_gemm(t, second, first, kMinusOne, t.alpha);
}

int trsm_device(const Trsm &t, cudaStream_t s, bool *emulated) {
    *emulated = false;
    if (t.M == 0 || t.N == 0) return BLASX_OK;
    if (t.alpha.re == 0 && t.alpha.im == 0) {  // X = 0; A is not read
        Gemm z;
        z.dt = t.dt;
        z.ta = z.tb = NoTrans;
        z.M = t.M; z.N = t.N; z.K = 0;
        z.alpha = cplx{0.0, 0.0}; z.beta = cplx{0.0, 0.0};
        z.A = nullptr; z.lda = 1; z.B = nullptr; z.ldb = 1;
        z.C = t.B; z.ldc = t.ldb;
        return launch_scale(z, s);
    }
    return solve(t, Range{0, t.order()}, t.alpha, s, emulated);
}

}  // namespace bx

namespace bx {

TrmmScratch trmm_scratch_sizes(const Trsm &t) {
    TrmmScratch w;
    const size_t es = elem_size(t.dt);
    w.ldt = t.left ? kTrmmLeaf : (t.M + 31) / 32 * 32;
    w.diag_bytes = size_t(kTrmmLeaf) * kTrmmLeaf * es;
    w.temp_bytes = size_t(w.ldt) * size_t(t.left ? t.N : kTrmmLeaf) * es;
    return w;
}

int trmm_part_into(const Trsm &t, void *dst, int64_t lo, int64_t hi, const TrmmScratch &w, cudaStream_t s,
                   bool *emulated) {
    return multiply_into(t, dst, Range{lo, hi}, w, s, emulated);
}

int trmm_update_into(const Trsm &t, void *dst, int64_t tgt_lo, int64_t tgt_hi, int64_t src_lo, int64_t src_hi,
                     cudaStream_t s, bool *emulated) {
    Gemm g = update_gemm(t, Range{tgt_lo, tgt_hi}, Range{src_lo, src_hi}, t.alpha, kOne);
    g.C = static_cast<char *>(dst) + (static_cast<char *>(g.C) - static_cast<char *>(t.B));
    BX_TRY(device_gemm(g, s));
    if (call_stats().path == 2) *emulated = true;
    return BLASX_OK;
}

Gemm trmm_top_update(const Trsm &t) {
    const Range all{0, t.order()};
    if (all.size() <= kTrmmLeaf) {
        Gemm g = update_gemm(t, all, all, t.alpha, kOne);
        g.K = 0;
        return g;
    }
    Range first, second;
    trmm_split(t, all, &first, &second);
    return update_gemm(t, first, second, t.alpha, kOne);
}

int trmm_device(const Trsm &t, const TrmmScratch &w, cudaStream_t s, bool *emulated) {
    *emulated = false;
    if (t.M == 0 || t.N == 0) return BLASX_OK;
    if (t.alpha.re == 0 && t.alpha.im == 0) {  // B = 0; A is not read
        Gemm z;
        z.dt = t.dt;
        z.ta = z.tb = NoTrans;
        z.M = t.M; z.N = t.N; z.K = 0;
        z.alpha = cplx{0.0, 0.0}; z.beta = cplx{0.0, 0.0};
        z.A = nullptr; z.lda = 1; z.B = nullptr; z.ldb = 1;
        z.C = t.B; z.ldc = t.ldb;
        return launch_scale(z, s);
    }
    return multiply(t, Range{0, t.order()}, w, s, emulated);
}

}  // namespace bx
