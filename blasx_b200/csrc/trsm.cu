// trsm.cu -- triangular solve with many right-hand sides on device operands
// (the compute of cblas_?trsm).
//
// op(A) X = alpha B (left) or X op(A) = alpha B (right) is solved by
// recursive halving of the order-K triangle: solve the first half, update
// the second half's right-hand sides with one GEMM (device_gemm: native, or
// emulated on the INT8 tensor cores where the precision mode selects it),
// solve the second half. The top-level updates carry most of the K^2 * (M or
// N) work with K up to K/2, the shape the emulated GEMM needs; blocks of at
// most kLeaf rows are solved by substitution in one kernel.
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

constexpr int kLeaf = 64;                      // order of a substitution block
constexpr int kVecs = 64;                      // right-hand-side vectors per CTA
constexpr int kGroups = 4;                     // thread (v, g) owns rows g, g + 4, ...
constexpr int kRows = kLeaf / kGroups;         // rows per thread
constexpr int kThreads = kVecs * kGroups;

template <typename T> __device__ inline T negate(T a) { return -a; }
template <> __device__ inline z2 negate<z2>(z2 a) { return {-a.re, -a.im}; }
template <> __device__ inline c2 negate<c2>(c2 a) { return {-a.re, -a.im}; }

// Solves S x = c for nvec vectors at once, S the bs x bs (bs <= kLeaf)
// system matrix of one diagonal block: S = op(A_block) for a left solve, the
// transpose of op(A_block) for a right solve (x op(A) = c is op(A)^T x^T =
// c^T). S[i][k] is A[i + k lda] (s_trans = 0) or A[k + i lda] (s_trans = 1),
// conjugated when s_conj. S is lower (forward substitution) or upper
// (backward); only that triangle of S, and its diagonal unless unit, is read.
// Vector v, element i: left: C[i + v ldc] (columns of B); right: C[v + i ldc]
// (rows of B). Each vector is scaled by `scale` (alpha) on load.
//
// Thread (v, g) keeps elements g, g + 4, ... of vector v in registers. Step k
// (in substitution order): the owner of element k divides by the diagonal
// and publishes x_k in xs[k & 1][v]; after one barrier every thread applies
// c_i -= S[i][k] x_k to its later elements. The two xs rows alternate, so the
// write of step k + 1 never meets a read of step k (those finished before
// the barrier of step k + 1).
template <typename T>
__global__ void __launch_bounds__(kThreads)
    trsm_leaf_kernel(const T *__restrict__ A, int64_t lda, T *__restrict__ C, int64_t ldc, int bs,
                     int64_t nvec, int left, int s_trans, int s_conj, int unit, int forward, T scale) {
    using Ar = Arith<T>;
    extern __shared__ __align__(16) unsigned char smem[];
    T *S = reinterpret_cast<T *>(smem);  // S[i * kLeaf + k]
    T *xs = S + kLeaf * kLeaf;           // xs[buf * kVecs + v]
    const int tid = threadIdx.x;
    const int v = tid % kVecs, g = tid / kVecs;
    const int64_t vg = int64_t(blockIdx.x) * kVecs + v;
    const bool live = vg < nvec;

    for (int e = tid; e < bs * bs; e += kThreads) {
        const int i = e % bs, k = e / bs;
        const bool used = forward ? i > k : i < k;
        T val = Ar::zero();
        if (used || (i == k && !unit)) {
            val = s_trans ? A[k + int64_t(i) * lda] : A[i + int64_t(k) * lda];
            if (s_conj) val = Ar::conj(val);
        }
        S[i * kLeaf + k] = val;
    }
    T c[kRows];
#pragma unroll
    for (int m = 0; m < kRows; ++m) {
        const int i = g + kGroups * m;
        c[m] = Ar::zero();
        if (live && i < bs) c[m] = Ar::mul(scale, left ? C[i + vg * ldc] : C[vg + int64_t(i) * ldc]);
    }
    __syncthreads();

    for (int step = 0; step < bs; ++step) {
        const int k = forward ? step : bs - 1 - step;
        T *xb = xs + (step & 1) * kVecs;
        if (g == k % kGroups) {
            const int mk = k / kGroups;
#pragma unroll
            for (int m = 0; m < kRows; ++m)
                if (m == mk) {
                    T x = c[m];
                    if (!unit) x = quot(x, S[k * kLeaf + k]);
                    c[m] = x;
                    xb[v] = x;
                }
        }
        __syncthreads();
        const T xk = xb[v];
#pragma unroll
        for (int m = 0; m < kRows; ++m) {
            const int i = g + kGroups * m;
            if (i < bs && (forward ? i > k : i < k)) c[m] = Ar::fma(negate(S[i * kLeaf + k]), xk, c[m]);
        }
    }
    if (!live) return;
#pragma unroll
    for (int m = 0; m < kRows; ++m) {
        const int i = g + kGroups * m;
        if (i < bs) (left ? C[i + vg * ldc] : C[vg + int64_t(i) * ldc]) = c[m];
    }
}

template <typename T> size_t leaf_smem() { return sizeof(T) * (kLeaf * kLeaf + 2 * kVecs); }

template <typename T>
int launch_leaf_t(const Trsm &t, int64_t lo, int64_t hi, cplx scale, int s_trans, int forward, cudaStream_t s) {
    static bool attr_set = false;
    if (!attr_set) {
        BX_CUDA(cudaFuncSetAttribute(trsm_leaf_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(leaf_smem<T>())));
        attr_set = true;
    }
    const int64_t nvec = t.left ? t.N : t.M;
    const T *A = static_cast<const T *>(t.A) + lo + lo * t.lda;
    T *C = static_cast<T *>(t.B) + (t.left ? lo : lo * t.ldb);
    const int64_t blocks = (nvec + kVecs - 1) / kVecs;
    if (blocks > 0x7fffffff) return set_error(BLASX_ERR_UNSUPPORTED, "trsm: too many right-hand sides");
    const bool conj = is_complex(t.dt) && t.trans == ConjT;
    trsm_leaf_kernel<T><<<unsigned(blocks), kThreads, leaf_smem<T>(), s>>>(
        A, t.lda, C, t.ldb, int(hi - lo), nvec, t.left, s_trans, conj, t.unit, forward, from_cplx<T>(scale));
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
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
// kLeaf rows.
void split(const Trsm &t, Range r, Range *first, Range *second) {
    const int64_t n = r.size();
    const int64_t half = std::min(n - 1, (n / 2 + kLeaf - 1) / kLeaf * kLeaf);
    if (forward_of(t)) {
        *first = {r.lo, r.lo + half};
        *second = {r.lo + half, r.hi};
    } else {
        *first = {r.hi - half, r.hi};
        *second = {r.lo, r.hi - half};
    }
}

// B[tgt] = scale B[tgt] - op(A)[tgt, src] X[src] (left) or
// B[:, tgt] = scale B[:, tgt] - X[:, src] op(A)[src, tgt] (right).
Gemm update_gemm(const Trsm &t, Range tgt, Range src, cplx scale) {
    const size_t es = elem_size(t.dt);
    const char *A = static_cast<const char *>(t.A);
    char *B = static_cast<char *>(t.B);
    const int tr = (t.trans == ConjT && !is_complex(t.dt)) ? TransT : t.trans;
    Gemm g;
    g.dt = t.dt;
    g.alpha = cplx{-1.0, 0.0};
    g.beta = scale;
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

int solve(const Trsm &t, Range r, cplx scale, cudaStream_t s, bool *emulated) {
    if (r.size() <= kLeaf) return launch_leaf(t, r.lo, r.hi, scale, s_trans_of(t), forward_of(t), s);
    Range first, second;
    split(t, r, &first, &second);
    BX_TRY(solve(t, first, scale, s, emulated));
    BX_TRY(device_gemm(update_gemm(t, second, first, scale), s));
    if (call_stats().path == 2) *emulated = true;
    return solve(t, second, cplx{1.0, 0.0}, s, emulated);
}

}  // namespace

Gemm trsm_top_update(const Trsm &t) {
    const Range all{0, t.order()};
    if (all.size() <= kLeaf) {
        Gemm g = update_gemm(t, all, all, t.alpha);
        g.K = 0;
        return g;
    }
    Range first, second;
    split(t, all, &first, &second);
    return update_gemm(t, second, first, t.alpha);
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
