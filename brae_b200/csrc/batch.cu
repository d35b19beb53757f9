// batch.cu -- the batched PCG + GAMG solve of many independent cases (batch.cuh): descriptor tables,
// tile lists, the batched kernels and the solve loop, one CUDA graph per iteration.
//
// Every kernel here is the single-case kernel of ldu_kernels.cuh / solver.cu applied to a tile of
// one case's cells, with the same per-cell arithmetic; only the reductions are shaped per tile
// (2048 cells) and then per case, in a fixed order.
//
// Reference: GAMG = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu
#include "batch.cuh"
#include "pipe_kernels.cuh"
#include "capi_internal.cuh"

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <mutex>

namespace b2g {

namespace {

constexpr int BT = 256;       // threads per tile block
constexpr int kTile = 2048;   // cells per tile
constexpr int kWarpsPerBlock = BT / 32;

int warpGrid(int n) { return std::max(1, ceilDiv(n, kWarpsPerBlock)); }

template <class T>
__device__ __forceinline__ bool inactive(const SegLevel<T>& s, const int* active)
{
    return active && active[s.caseIdx] == 0;
}

// ---------------------------------------------------------------------------------------------
// row and element-wise kernels (one block per tile)
// ---------------------------------------------------------------------------------------------

// lduMatrix::Amul (GAMG:62-88)
template <class T>
__global__ void __launch_bounds__(BT) bAmul(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                            int rx, int ry, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    const k::Rows<T> A = s.rows;
    const T* __restrict__ x = s.v[rx];
    T* __restrict__ y = s.v[ry];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
    {
        T acc = mulRn(A.diag[c], x[c]);
        const int e1 = A.rowStart[c + 1];
        for (int e = A.rowStart[c]; e < e1; ++e) acc = addRn(acc, mulRn(A.val[e], x[A.col[e]]));
        y[c] = acc;
    }
}

// lduMatrix::residual (GAMG:90-117); r may alias the source
template <class T>
__global__ void __launch_bounds__(BT) bResidual(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                                int rsrc, int rpsi, int rr, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    const k::Rows<T> A = s.rows;
    const T* src = s.v[rsrc];
    const T* __restrict__ psi = s.v[rpsi];
    T* r = s.v[rr];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
    {
        T acc = subRn(src[c], mulRn(A.diag[c], psi[c]));
        const int e1 = A.rowStart[c + 1];
        for (int e = A.rowStart[c]; e < e1; ++e) acc = subRn(acc, mulRn(A.val[e], psi[A.col[e]]));
        r[c] = acc;
    }
}

// r = a - b
template <class T>
__global__ void __launch_bounds__(BT) bSubtract(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                                int ra, int rb, int rr, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    const T* __restrict__ a = s.v[ra];
    const T* __restrict__ b = s.v[rb];
    T* __restrict__ r = s.v[rr];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT) r[c] = subRn(a[c], b[c]);
}

template <class T>
__global__ void __launch_bounds__(BT) bZero(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                            int rx, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    T* __restrict__ x = s.v[rx];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT) x[c] = T(0);
}

// psi += corr
template <class T>
__global__ void __launch_bounds__(BT) bAdd(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                           int rpsi, int rcorr, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    T* __restrict__ psi = s.v[rpsi];
    const T* __restrict__ corr = s.v[rcorr];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT) psi[c] = addRn(psi[c], corr[c]);
}

template <class T>
__global__ void __launch_bounds__(BT) bCopy(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                            int rdst, int rsrc, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    T* __restrict__ d = s.v[rdst];
    const T* __restrict__ x = s.v[rsrc];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT) d[c] = x[c];
}

// out (type T) = in (type S), same tiles and descriptors in both tables
template <class T, class S>
__global__ void __launch_bounds__(BT) bCast(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ out,
                                            const SegLevel<S>* __restrict__ in, int rout, int rin,
                                            const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& so = out[t.x];
    if (inactive(so, active)) return;
    T* __restrict__ o = so.v[rout];
    const S* __restrict__ x = in[t.x].v[rin];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT) o[c] = static_cast<T>(x[c]);
}

// natural cell order <-> position order (toPos: out[i] = in[posCell[i]]; else out[posCell[i]] = in[i])
__global__ void __launch_bounds__(BT) bPermute(const int4* __restrict__ tiles, const SegLevel<double>* __restrict__ segs,
                                               int rin, int rout, int toPos)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<double>& s = segs[t.x];
    const int* __restrict__ pc = s.posCell;
    const double* __restrict__ in = s.v[rin];
    double* __restrict__ out = s.v[rout];
    for (int i = t.y + threadIdx.x; i < t.z; i += BT)
    {
        if (toPos) out[i] = in[pc[i]];
        else out[pc[i]] = in[i];
    }
}

// restrictField (GAMG:410-419): tiles over the next level's cells, t.x the fine descriptor
template <class T>
__global__ void __launch_bounds__(BT) bRestrict(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                                int rf, int rc, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& f = segs[t.x];
    if (inactive(f, active)) return;
    const T* __restrict__ ff = f.v[rf];
    T* __restrict__ cf = segs[f.coarseSeg].v[rc];
    const int* __restrict__ rs = f.rStartP;
    const int* __restrict__ rl = f.rListP;
    for (int C = t.y + threadIdx.x; C < t.z; C += BT)
    {
        T acc = T(0);
        const int e1 = rs[C + 1];
        for (int e = rs[C]; e < e1; ++e) acc = addRn(acc, ff[rl[e]]);
        cf[C] = acc;
    }
}

// prolongField (GAMG:422-432): tiles over the fine level's cells
template <class T>
__global__ void __launch_bounds__(BT) bProlong(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                               int rc, int rf, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& f = segs[t.x];
    if (inactive(f, active)) return;
    const T* __restrict__ cf = segs[f.coarseSeg].v[rc];
    T* __restrict__ ff = f.v[rf];
    const int* __restrict__ map = f.prolongP;
    for (int i = t.y + threadIdx.x; i < t.z; i += BT) ff[i] = cf[map[i]];
}

// one colour of a multicolour Gauss-Seidel sweep of the FP32 V-cycle: tiles of one colour's rows
__global__ void __launch_bounds__(BT) bMcSweep(const int4* __restrict__ tiles, const SegLevel<float>* __restrict__ segs,
                                               int rpsi, int rsrc, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<float>& s = segs[t.x];
    if (inactive(s, active)) return;
    const int* __restrict__ pos = s.mcPos;
    const int* __restrict__ slice = s.mcSlice;
    const int* __restrict__ col = s.mcCol;
    const float* __restrict__ val = s.mcVal;
    const float* __restrict__ diag = s.mcDiag;
    const float* __restrict__ b = s.v[rsrc];
    float* __restrict__ psi = s.v[rpsi];
    for (int r = t.y + threadIdx.x; r < t.z; r += BT) k::mcRowUpdate(r, pos, slice, col, val, diag, b, psi);
}

// every sweep of one small case's multicolour smoothing in one block (block i: descriptor cases[i])
__global__ void __launch_bounds__(1024) bMcSmoothSmall(const int* __restrict__ cases,
                                                       const SegLevel<float>* __restrict__ segs, int rpsi, int rsrc,
                                                       int nSweeps, const int* __restrict__ active)
{
    const SegLevel<float>& s = segs[cases[blockIdx.x]];
    if (inactive(s, active)) return;
    const int* __restrict__ pos = s.mcPos;
    const int* __restrict__ slice = s.mcSlice;
    const int* __restrict__ col = s.mcCol;
    const float* __restrict__ val = s.mcVal;
    const float* __restrict__ diag = s.mcDiag;
    const int* __restrict__ cs = s.mcColourStart;
    const int nColours = s.mcColours;
    const float* __restrict__ b = s.v[rsrc];
    float* __restrict__ psi = s.v[rpsi];
    for (int sw = 0; sw < nSweeps; ++sw)
        for (int c = 0; c < nColours; ++c)
        {
            const int end = cs[c + 1];
            for (int r = cs[c] + threadIdx.x; r < end; r += blockDim.x)
                k::mcRowUpdate(r, pos, slice, col, val, diag, b, psi);
            __syncthreads();
        }
}

// ---------------------------------------------------------------------------------------------
// scale (GAMG:386-407), per case
// ---------------------------------------------------------------------------------------------

template <class T>
__global__ void __launch_bounds__(BT) bAmulScaleDots(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                                     int rfield, int rsrc, int racf, T* __restrict__ partial,
                                                     const int* __restrict__ active)
{
    __shared__ T sh[BT / 32];
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    const k::Rows<T> A = s.rows;
    const T* __restrict__ field = s.v[rfield];
    const T* __restrict__ source = s.v[rsrc];
    T* __restrict__ Acf = s.v[racf];
    T num = T(0), den = T(0);
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
    {
        const T fc = field[c];
        T acc = mulRn(A.diag[c], fc);
        const int e1 = A.rowStart[c + 1];
        for (int e = A.rowStart[c]; e < e1; ++e) acc = addRn(acc, mulRn(A.val[e], field[A.col[e]]));
        Acf[c] = acc;
        num = addRn(num, mulRn(fc, source[c]));
        den = addRn(den, mulRn(fc, acc));
    }
    num = k::blockSum<T, BT>(num, sh);
    den = k::blockSum<T, BT>(den, sh);
    if (threadIdx.x == 0)
    {
        partial[2 * blockIdx.x] = num;
        partial[2 * blockIdx.x + 1] = den;
    }
}

template <class T>
__device__ __forceinline__ T warpSum(T v)
{
    for (int o = 16; o > 0; o >>= 1) v = addRn(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;  // valid in lane 0
}

// sf per listed case from its tiles' partials (one warp per case)
template <class T>
__global__ void __launch_bounds__(BT) bScaleFactor(const int* __restrict__ segOf, const int* __restrict__ tileStart,
                                                   int nSeg, const SegLevel<T>* __restrict__ segs,
                                                   const T* __restrict__ partial, T* __restrict__ sf,
                                                   const int* __restrict__ active)
{
    const int ls = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (ls >= nSeg || inactive(segs[segOf[ls]], active)) return;
    T num = T(0), den = T(0);
    for (int i = tileStart[ls] + lane; i < tileStart[ls + 1]; i += 32)
    {
        num = addRn(num, partial[2 * i]);
        den = addRn(den, partial[2 * i + 1]);
    }
    num = warpSum(num);
    den = warpSum(den);
    if (lane == 0)
    {
        const T v = k::Small<T>::vsmall;
        sf[ls] = divRn(num, den >= T(0) ? addRn(den, v) : subRn(den, v));
    }
}

// scale's sums in the reference's serial order (one warp per listed case; FP64)
__global__ void __launch_bounds__(BT) bSerialScaleDots(const int* __restrict__ segOf, int nSeg,
                                                       const SegLevel<double>* __restrict__ segs, int rfield, int rsrc,
                                                       int racf, double* __restrict__ sf, const int* __restrict__ active)
{
    const int ls = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (ls >= nSeg) return;
    const SegLevel<double>& s = segs[segOf[ls]];
    if (inactive(s, active)) return;
    const int n = s.rows.n;
    const int* __restrict__ posOf = s.posOf;
    const double* __restrict__ field = s.v[rfield];
    const double* __restrict__ source = s.v[rsrc];
    const double* __restrict__ Acf = s.v[racf];
    double num = 0.0, den = 0.0;
    for (int base = 0; base < n; base += 32)
    {
        const int c = base + lane;
        double tn = 0.0, td = 0.0;
        if (c < n)
        {
            const int i = posOf[c];
            tn = __dmul_rn(field[i], source[i]);
            td = __dmul_rn(field[i], Acf[i]);
        }
        const int cnt = min(32, n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double vn = __shfl_sync(0xffffffffu, tn, j);
            const double vd = __shfl_sync(0xffffffffu, td, j);
            if (lane == 0)
            {
                num = __dadd_rn(num, vn);
                den = __dadd_rn(den, vd);
            }
        }
    }
    if (lane == 0)
        sf[ls] = __ddiv_rn(num, den >= 0.0 ? __dadd_rn(den, k::Small<double>::vsmall)
                                           : __dsub_rn(den, k::Small<double>::vsmall));
}

// field = sf*field + (source - sf*Acf)/diag; t.w is the case's index in the list (its sf)
template <class T>
__global__ void __launch_bounds__(BT) bScaleUpdate(const int4* __restrict__ tiles, const SegLevel<T>* __restrict__ segs,
                                                   const T* __restrict__ sfs, int rfield, int rsrc, int racf,
                                                   const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    const T sf = sfs[t.w];
    T* __restrict__ field = s.v[rfield];
    const T* __restrict__ source = s.v[rsrc];
    const T* __restrict__ Acf = s.v[racf];
    const T* __restrict__ diag = s.rows.diag;
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
        field[c] = addRn(mulRn(sf, field[c]), divRn(subRn(source[c], mulRn(sf, Acf[c])), diag[c]));
}

// the finest level's scale update fused with psi += correction (GAMG:716-723)
template <class T>
__global__ void __launch_bounds__(BT) bScaleUpdateAdd(const int4* __restrict__ tiles,
                                                      const SegLevel<T>* __restrict__ segs, const T* __restrict__ sfs,
                                                      int rfield, int rsrc, int racf, int rpsi,
                                                      const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<T>& s = segs[t.x];
    if (inactive(s, active)) return;
    const T sf = sfs[t.w];
    const T* __restrict__ field = s.v[rfield];
    const T* __restrict__ source = s.v[rsrc];
    const T* __restrict__ Acf = s.v[racf];
    const T* __restrict__ diag = s.rows.diag;
    T* __restrict__ psi = s.v[rpsi];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
    {
        const T corr = addRn(mulRn(sf, field[c]), divRn(subRn(source[c], mulRn(sf, Acf[c])), diag[c]));
        psi[c] = addRn(psi[c], corr);
    }
}

// ---------------------------------------------------------------------------------------------
// finest-level reductions into each case's PCG scalars (FP64)
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ double& member(PcgScalars* s, size_t off)
{
    return *reinterpret_cast<double*>(reinterpret_cast<char*>(s) + off);
}

template <int OP>
__global__ void __launch_bounds__(BT) bReducePartial(const int4* __restrict__ tiles,
                                                     const SegLevel<double>* __restrict__ segs, int ra, int rb,
                                                     double* __restrict__ partial, const int* __restrict__ active)
{
    __shared__ double sh[BT / 32];
    const int4 t = tiles[blockIdx.x];
    const SegLevel<double>& s = segs[t.x];
    if (inactive(s, active)) return;
    const double* __restrict__ a = s.v[ra];
    const double* __restrict__ b = rb >= 0 ? s.v[rb] : nullptr;
    double acc = 0.0;
    for (int i = t.y + threadIdx.x; i < t.z; i += BT)
    {
        if (OP == k::RED_DOT) acc = __dadd_rn(acc, __dmul_rn(a[i], b[i]));
        else if (OP == k::RED_SUMMAG) acc = __dadd_rn(acc, fabs(a[i]));
        else acc = __dadd_rn(acc, a[i]);
    }
    acc = k::blockSum<double, BT>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// per listed case: the sum of its tiles' partials into its scalars at byte offset `off`
__global__ void __launch_bounds__(BT) bReduceFinal(const int* __restrict__ segOf, const int* __restrict__ tileStart,
                                                   int nSeg, const SegLevel<double>* __restrict__ segs,
                                                   const double* __restrict__ partial, size_t off,
                                                   const int* __restrict__ active)
{
    const int ls = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (ls >= nSeg) return;
    const SegLevel<double>& s = segs[segOf[ls]];
    if (inactive(s, active)) return;
    double v = 0.0;
    for (int i = tileStart[ls] + lane; i < tileStart[ls + 1]; i += 32) v = __dadd_rn(v, partial[i]);
    v = warpSum(v);
    if (lane == 0) member(s.scal, off) = v;
}

// the reference's serial order (one warp per listed case)
template <int OP>
__global__ void __launch_bounds__(BT) bSerialReduce(const int* __restrict__ segOf, int nSeg,
                                                    const SegLevel<double>* __restrict__ segs, int ra, int rb,
                                                    size_t off, const int* __restrict__ active)
{
    const int ls = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (ls >= nSeg) return;
    const SegLevel<double>& s = segs[segOf[ls]];
    if (inactive(s, active)) return;
    const int n = s.rows.n;
    const int* __restrict__ posOf = s.posOf;
    const double* __restrict__ a = s.v[ra];
    const double* __restrict__ b = rb >= 0 ? s.v[rb] : nullptr;
    double acc = 0.0;
    for (int base = 0; base < n; base += 32)
    {
        const int c = base + lane;
        double term = 0.0;
        if (c < n)
        {
            const int i = posOf[c];
            if (OP == k::RED_DOT) term = __dmul_rn(a[i], b[i]);
            else if (OP == k::RED_SUMMAG) term = fabs(a[i]);
            else term = a[i];
        }
        const int cnt = min(32, n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double v = __shfl_sync(0xffffffffu, term, j);
            if (lane == 0) acc = __dadd_rn(acc, v);
        }
    }
    if (lane == 0) member(s.scal, off) = acc;
}

// normFactor's per-cell summand (GAMG:119-159), xRef from the case's sumPsi
__global__ void __launch_bounds__(BT) bNormFactorPartial(const int4* __restrict__ tiles,
                                                         const SegLevel<double>* __restrict__ segs, int rpsi, int rsrc,
                                                         int rapsi, double* __restrict__ partial)
{
    __shared__ double sh[BT / 32];
    const int4 t = tiles[blockIdx.x];
    const SegLevel<double>& s = segs[t.x];
    const k::Rows<double> A = s.rows;
    const double* __restrict__ source = s.v[rsrc];
    const double* __restrict__ Apsi = s.v[rapsi];
    (void)rpsi;
    const double xRef = __ddiv_rn(s.scal->sumPsi, static_cast<double>(A.n));
    double acc = 0.0;
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
    {
        double sumA = A.diag[c];
        const int e1 = A.rowStart[c + 1];
        for (int e = A.rowStart[c]; e < e1; ++e) sumA = __dadd_rn(sumA, A.val[e]);
        const double tt = __dmul_rn(sumA, xRef);
        acc = __dadd_rn(acc, __dadd_rn(fabs(__dsub_rn(Apsi[c], tt)), fabs(__dsub_rn(source[c], tt))));
    }
    acc = k::blockSum<double, BT>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// normFactor in the reference's serial order (one warp per listed case), + 1e-20 included
__global__ void __launch_bounds__(BT) bSerialNormFactor(const int* __restrict__ segOf, int nSeg,
                                                        const SegLevel<double>* __restrict__ segs, int rpsi, int rsrc,
                                                        int rapsi)
{
    const int ls = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (ls >= nSeg) return;
    const SegLevel<double>& s = segs[segOf[ls]];
    const k::Rows<double> A = s.rows;
    const int* __restrict__ posOf = s.posOf;
    const double* __restrict__ psi = s.v[rpsi];
    const double* __restrict__ source = s.v[rsrc];
    const double* __restrict__ Apsi = s.v[rapsi];
    double sumPsi = 0.0;
    for (int base = 0; base < A.n; base += 32)
    {
        const int i = base + lane;
        const double v = i < A.n ? psi[posOf[i]] : 0.0;
        const int cnt = min(32, A.n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double w = __shfl_sync(0xffffffffu, v, j);
            if (lane == 0) sumPsi = __dadd_rn(sumPsi, w);
        }
    }
    const double xRef = __ddiv_rn(__shfl_sync(0xffffffffu, sumPsi, 0), static_cast<double>(A.n));
    double acc = 0.0;
    for (int base = 0; base < A.n; base += 32)
    {
        const int c = base + lane;
        double term = 0.0;
        if (c < A.n)
        {
            const int i = posOf[c];
            double sumA = A.diag[i];
            for (int e = A.rowStart[i]; e < A.rowStart[i + 1]; ++e) sumA = __dadd_rn(sumA, A.val[e]);
            const double tt = __dmul_rn(sumA, xRef);
            term = __dadd_rn(fabs(__dsub_rn(Apsi[i], tt)), fabs(__dsub_rn(source[i], tt)));
        }
        const int cnt = min(32, A.n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double v = __shfl_sync(0xffffffffu, term, j);
            if (lane == 0) acc = __dadd_rn(acc, v);
        }
    }
    if (lane == 0) s.scal->nf = __dadd_rn(acc, 1e-20);
}

// ---------------------------------------------------------------------------------------------
// PCG (PCG.C; gamg_solver_cpp.cu:1031-1143), per case
// ---------------------------------------------------------------------------------------------

constexpr double kSmall = 1e-20;
constexpr double kVSmall = 1e-300;
constexpr double kGreat = 1e+20;

__device__ __forceinline__ bool convergedD(double fin, double init, double tol, double relTol)
{
    return fin < tol || (relTol > kSmall && fin < __dmul_rn(relTol, init));
}

// Level-0 descriptors are the first K of the table, in case order.
__global__ void bNfFinish(int K, const SegLevel<double>* __restrict__ segs)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < K) segs[c].scal->nf = __dadd_rn(segs[c].scal->nf, kSmall);
}

// the initial residual, and which cases iterate at all
__global__ void bStart(int K, const SegLevel<double>* __restrict__ segs, double tol, double relTol, int minIter,
                       int* __restrict__ active, int* __restrict__ nActive)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K) return;
    PcgScalars* s = segs[c].scal;
    const double init = __ddiv_rn(s->sumMag, s->nf);
    s->initRes = init;
    s->finalRes = init;
    s->wArA = kGreat;
    s->wArAold = kGreat;
    s->iter = 0;
    s->singular = 0;
    const int go = (minIter <= 0 && convergedD(init, init, tol, relTol)) ? 0 : 1;
    active[c] = go;
    if (go) atomicAdd(nActive, 1);
}

__global__ void __launch_bounds__(BT) bPUpdate(const int4* __restrict__ tiles, const SegLevel<double>* __restrict__ segs,
                                               int rw, int rp, int flexible, const int* __restrict__ active)
{
    const int4 t = tiles[blockIdx.x];
    const SegLevel<double>& sg = segs[t.x];
    if (inactive(sg, active)) return;
    const PcgScalars* s = sg.scal;
    const int iter = s->iter;
    double beta = 0.0;
    if (iter != 0)
    {
        if (flexible)
        {
            const double d = s->wArAold;
            beta = (d > 1e-300 || d < -1e-300) ? fmax(0.0, __ddiv_rn(__dsub_rn(s->wArA, s->wrOld), d)) : 0.0;
        }
        else
        {
            beta = __ddiv_rn(s->wArA, s->wArAold);
        }
    }
    const double* __restrict__ w = sg.v[rw];
    double* __restrict__ p = sg.v[rp];
    for (int c = t.y + threadIdx.x; c < t.z; c += BT) p[c] = iter == 0 ? w[c] : __dadd_rn(w[c], __dmul_rn(beta, p[c]));
}

// checkSingularity, then psi += alpha*p, r -= alpha*w with the tiles' sums of |r|
__global__ void __launch_bounds__(BT) bAlphaUpdate(const int4* __restrict__ tiles,
                                                   const SegLevel<double>* __restrict__ segs, int rpsi, int rp, int rr,
                                                   int rw, int rold, double* __restrict__ partial,
                                                   const int* __restrict__ active)
{
    __shared__ double sh[BT / 32];
    const int4 t = tiles[blockIdx.x];
    const SegLevel<double>& sg = segs[t.x];
    if (inactive(sg, active)) return;
    PcgScalars* s = sg.scal;
    const double wApA = s->wApA;
    if (__ddiv_rn(fabs(wApA), s->nf) < kVSmall)
    {
        if (t.y == 0 && threadIdx.x == 0) s->singular = 1;
        if (threadIdx.x == 0) partial[blockIdx.x] = 0.0;
        return;
    }
    const double alpha = __ddiv_rn(s->wArA, wApA);
    double* __restrict__ psi = sg.v[rpsi];
    const double* __restrict__ p = sg.v[rp];
    double* __restrict__ r = sg.v[rr];
    const double* __restrict__ w = sg.v[rw];
    double* __restrict__ rOld = rold >= 0 ? sg.v[rold] : nullptr;
    double acc = 0.0;
    for (int c = t.y + threadIdx.x; c < t.z; c += BT)
    {
        const double rc = r[c];
        if (rOld) rOld[c] = rc;
        psi[c] = __dadd_rn(psi[c], __dmul_rn(alpha, p[c]));
        const double rn = __dsub_rn(rc, __dmul_rn(alpha, w[c]));
        r[c] = rn;
        acc = __dadd_rn(acc, fabs(rn));
    }
    acc = k::blockSum<double, BT>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// the end of an iteration: the residual, beta's memory and the count; then whether the case goes on
__global__ void bFinish(int K, const SegLevel<double>* __restrict__ segs, double tol, double relTol, int maxIter,
                        int minIter, int* __restrict__ active, int* __restrict__ nActive)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K || active[c] == 0) return;
    PcgScalars* s = segs[c].scal;
    if (s->singular)
    {
        active[c] = 0;
        return;
    }
    s->finalRes = __ddiv_rn(s->sumMag, s->nf);
    s->wArAold = s->wArA;
    s->iter += 1;
    const int go = ((s->iter < maxIter && !convergedD(s->finalRes, s->initRes, tol, relTol)) || s->iter < minIter)
                       ? 1 : 0;
    active[c] = go;
    if (go) atomicAdd(nActive, 1);
}

__global__ void bGatherPerf(int K, const SegLevel<double>* __restrict__ segs, BatchPerf* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K) return;
    const PcgScalars* s = segs[c].scal;
    out[c].initialResidual = s->initRes;
    out[c].finalResidual = s->finalRes;
    out[c].nIterations = s->iter;
    out[c].pad = 0;
}

// ---------------------------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------------------------

// tiles of kTile cells over each (descriptor, cell count) in order
void buildTiles(TileList& L, const std::vector<std::pair<int, int>>& segCells, cudaStream_t s)
{
    std::vector<int4> tiles;
    std::vector<int> segOf, tileStart;
    for (size_t i = 0; i < segCells.size(); ++i)
    {
        segOf.push_back(segCells[i].first);
        tileStart.push_back(static_cast<int>(tiles.size()));
        const int n = segCells[i].second;
        for (int b = 0; b < n; b += kTile)
            tiles.push_back(make_int4(segCells[i].first, b, std::min(n, b + kTile), static_cast<int>(i)));
    }
    tileStart.push_back(static_cast<int>(tiles.size()));
    L.nTiles = static_cast<int>(tiles.size());
    L.nSeg = static_cast<int>(segOf.size());
    if (!tiles.empty()) L.tiles.upload(tiles.data(), tiles.size(), s);
    if (!segOf.empty()) L.segOf.upload(segOf.data(), segOf.size(), s);
    L.tileStart.upload(tileStart.data(), tileStart.size(), s);
}

template <class T>
k::GsArgs<T> gsArgsOf(const LevelAddr& L, const LevelCoef<T>& C, const T* b, T* psi, unsigned* progress, int* err)
{
    const GsSchedule& G = L.gs;
    k::GsArgs<T> a{};
    a.nParts = G.nParts;
    a.maxCells = G.maxCells;
    a.maxEnt = G.maxEnt;
    a.maxGat = G.maxGat;
    a.ahead = G.ahead;
    a.nPadded = G.nPadded;
    a.partChunkStart = G.partChunkStart.p;
    a.partPosStart = G.partPosStart.p;
    a.chunkRec = reinterpret_cast<const int4*>(G.chunkRec.p);
    a.upStart = G.upStart.p;
    a.upList = G.upList.p;
    a.hasDown = G.hasDown.p;
    a.blob = C.blob.p;
    a.gatSrc = G.gatSrc.p;
    a.b = b;
    a.psi = psi;
    a.progress = progress;
    a.ticket = nullptr;  // the batched launch draws its tickets from the level's own counter
    a.items = 0;
    a.spinLimit = k::kSpinLimit;
    a.publish = 1;
    a.err = err;
    a.trace = nullptr;
    a.traceDepths = 0;
    return a;
}

}  // namespace

template <> SegLevel<double>* Batch::segs<double>() { return segD.p; }
template <> SegLevel<float>* Batch::segs<float>() { return segF.p; }

Batch::Batch(std::vector<Matrix*> cs, cudaStream_t s) : stream(s), cases(std::move(cs))
{
    const int K = static_cast<int>(cases.size());
    if (K < 1) fail(B2G_ERR_ARGUMENT, "b2g batch: no cases");
    int dev = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    {
        std::vector<Matrix*> sorted(cases);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
            fail(B2G_ERR_ARGUMENT, "b2g batch: a matrix appears twice (each case is one matrix)");
    }
    for (Matrix* A : cases)
    {
        if (!A) fail(B2G_ERR_ARGUMENT, "b2g batch: null case");
        if (A->mesh->device != dev) fail(B2G_ERR_ARGUMENT, "b2g batch: every case must live on the current device");
        if (A->coupled)
            fail(B2G_ERR_REFUSED, "b2g batch: a matrix with a coupled pair is solved alone (b2g_gamg_solve_coupled)");
        if (A->nLevels() == 0)
            fail(B2G_ERR_REFUSED, "b2g GAMG: no coarse levels created, either matrix too small for GAMG or "
                                  "nCellsInCoarsestLevel too large (GAMGSolver.C:333).");
        A->buildCoarse();
        A->ensureFp32();
        B2G_CUDA(cudaStreamSynchronize(A->stream));
        nLevelsOf.push_back(A->nLevels());
        maxLevels = std::max(maxLevels, A->nLevels());
    }
    // descriptors, level-major, cases in order within a level
    std::vector<SegLevel<double>> hD;
    std::vector<SegLevel<float>> hF;
    segOfCase.assign(K, std::vector<int>());
    for (int lv = 0; lv <= maxLevels; ++lv)
    {
        levelSeg0.push_back(static_cast<int>(hD.size()));
        for (int c = 0; c < K; ++c)
        {
            if (lv > nLevelsOf[c]) continue;
            Matrix& A = *cases[c];
            const LevelAddr& L = A.mesh->lev[lv];
            SegLevel<double> d{};
            SegLevel<float> f{};
            d.rows = k::Rows<double>{L.nCells, L.gs.posRow.p, L.gs.entColPos.p, A.v64.coef[lv].rowVal.p,
                                     A.v64.coef[lv].gsDiag.p};
            f.rows = k::Rows<float>{L.nCells, L.gs.posRow.p, L.gs.entColPos.p, A.v32.coef[lv].rowVal.p,
                                    A.v32.coef[lv].gsDiag.p};
            d.posOf = f.posOf = L.gs.posOf.p;
            d.posCell = f.posCell = L.gs.posCell.p;
            d.v[V_ACF] = A.v64.ACf.p;
            d.v[V_PRE] = A.v64.preSmoothed.p;
            f.v[V_ACF] = A.v32.ACf.p;
            f.v[V_PRE] = A.v32.preSmoothed.p;
            if (lv == 0)
            {
                d.v[V_W] = A.wA.p;
                d.v[V_R] = A.rA.p;
                d.v[V_AWA] = A.AwA.p;
                d.v[V_FC] = A.fc.p;
                d.v[V_FR] = A.fr.p;
                d.v[V_PSI] = A.psi.p;
                d.v[V_SOURCE] = A.source.p;
                d.v[V_P] = A.pA.p;
                d.v[V_ROLD] = A.rOld.p;
                f.v[V_W] = A.w32.p;
                f.v[V_R] = A.r32.p;
                f.v[V_AWA] = A.AwA32.p;
                f.v[V_FC] = A.fc32.p;
                f.v[V_FR] = A.fr32.p;
            }
            else
            {
                d.v[V_CORR] = A.v64.corr[lv - 1].p;
                d.v[V_SRC] = A.v64.src[lv - 1].p;
                f.v[V_CORR] = A.v32.corr[lv - 1].p;
                f.v[V_SRC] = A.v32.src[lv - 1].p;
            }
            d.coarseSeg = f.coarseSeg = -1;
            if (lv < nLevelsOf[c])
            {
                const Step& S = A.mesh->step[lv];
                d.nCoarse = f.nCoarse = S.nCoarse;
                d.rStartP = f.rStartP = S.rStartP.p;
                d.rListP = f.rListP = S.rListP.p;
                d.prolongP = f.prolongP = S.prolongP.p;
            }
            d.scal = f.scal = A.scal.p;
            d.caseIdx = f.caseIdx = c;
            segOfCase[c].push_back(static_cast<int>(hD.size()));
            hD.push_back(d);
            hF.push_back(f);
        }
    }
    levelSeg0.push_back(static_cast<int>(hD.size()));
    for (int c = 0; c < K; ++c)
        for (int lv = 0; lv < nLevelsOf[c]; ++lv)
            hD[segOfCase[c][lv]].coarseSeg = hF[segOfCase[c][lv]].coarseSeg = segOfCase[c][lv + 1];
    segD.upload(hD.data(), hD.size(), stream);
    segF.upload(hF.data(), hF.size(), stream);
    hostF = hF;
    err.alloc(1, stream);
    err.zero(stream);
    // tile lists and the Gauss-Seidel launch of each level
    int maxTiles = 1;
    lev.resize(maxLevels + 1);
    for (int lv = 0; lv <= maxLevels; ++lv)
    {
        BatchLevel& B = lev[lv];
        std::vector<std::pair<int, int>> all, up, sc, down;
        for (int c = 0; c < K; ++c)
        {
            if (lv > nLevelsOf[c]) continue;
            const int sg = segOfCase[c][lv];
            const int n = cases[c]->n(lv);
            all.emplace_back(sg, n);
            if (nLevelsOf[c] >= lv + 1)
            {
                up.emplace_back(sg, n);
                down.emplace_back(sg, cases[c]->n(lv + 1));
            }
            if (lv >= 1 && nLevelsOf[c] >= lv + 2) sc.emplace_back(sg, n);
        }
        buildTiles(B.all, all, stream);
        buildTiles(B.up, up, stream);
        buildTiles(B.scale, sc, stream);
        buildTiles(B.down, down, stream);
        maxTiles = std::max({maxTiles, B.all.nTiles, B.up.nTiles, B.scale.nTiles, B.down.nTiles});
        // the sweep: the up cases (level 0: every case)
        std::vector<k::GsArgs<double>> g64;
        std::vector<k::GsArgs<float>> g32;
        std::vector<int4> parts;
        std::vector<int> partBase;
        int maxM = 0;
        int totalParts = 0;
        for (int c = 0; c < K; ++c)
        {
            if (nLevelsOf[c] < lv + 1 || lv > nLevelsOf[c]) continue;
            const LevelAddr& L = cases[c]->mesh->lev[lv];
            if (L.nCells == 0) continue;
            partBase.push_back(totalParts);
            totalParts += L.gs.nParts;
        }
        // the parts' progress lines, then one line for the launch's ticket counter
        B.progress.alloc((static_cast<size_t>(totalParts) + 1) * k::kProgressStride, stream);
        B.progress.zero(stream);
        B.ticketAt = static_cast<size_t>(totalParts) * k::kProgressStride;
        int pb = 0;
        for (int c = 0; c < K; ++c)
        {
            if (nLevelsOf[c] < lv + 1 || lv > nLevelsOf[c]) continue;
            Matrix& A = *cases[c];
            const LevelAddr& L = A.mesh->lev[lv];
            if (L.nCells == 0) continue;
            const GsSchedule& G = L.gs;
            unsigned* prog = B.progress.p + static_cast<size_t>(partBase[pb++]) * k::kProgressStride;
            const double* b64 = lv == 0 ? A.rA.p : A.v64.src[lv - 1].p;
            double* x64 = lv == 0 ? A.wA.p : A.v64.corr[lv - 1].p;
            const float* b32 = lv == 0 ? A.r32.p : A.v32.src[lv - 1].p;
            float* x32 = lv == 0 ? A.w32.p : A.v32.corr[lv - 1].p;
            const int arg = static_cast<int>(g64.size());
            g64.push_back(gsArgsOf<double>(L, A.v64.coef[lv], b64, x64, prog, err.p));
            g32.push_back(gsArgsOf<float>(L, A.v32.coef[lv], b32, x32, prog, err.p));
            for (int q = 0; q < G.nParts; ++q) parts.push_back(make_int4(arg, q, c, 0));
            maxM = std::max(maxM, G.maxCells);
            B.smem64 = std::max(B.smem64, k::gsSmemBytes<double>(G.maxCells, G.maxEnt, G.maxGat));
            B.smem32 = std::max(B.smem32, k::gsSmemBytes<float>(G.maxCells, G.maxEnt, G.maxGat));
        }
        B.nParts = static_cast<int>(parts.size());
        B.block = maxM + 128;
        B.hostParts = parts;
        if (!parts.empty())
        {
            B.gs64.upload(g64.data(), g64.size(), stream);
            B.gs32.upload(g32.data(), g32.size(), stream);
            B.parts.upload(parts.data(), parts.size(), stream);
        }
    }
    {
        std::vector<std::pair<int, int>> co;
        std::vector<k::CoarsestArgs<double>> args;
        for (int c = 0; c < K; ++c)
        {
            Matrix& A = *cases[c];
            const int lv = nLevelsOf[c];
            const LevelAddr& L = A.mesh->lev[lv];
            co.emplace_back(segOfCase[c][lv], L.nCells);
            k::CoarsestArgs<double> a{};
            a.n = L.nCells;
            a.nF = L.nFaces;
            a.lower = L.lower.p;
            a.upper = L.upper.p;
            a.posOf = L.gs.posOf.p;
            a.rowStart = L.gs.posRow.p;
            a.col = L.gs.entColPos.p;
            a.val = A.v64.coef[lv].rowVal.p;
            a.diag = A.v64.coef[lv].gsDiag.p;
            a.coef = A.v64.coef[lv].upper.p;
            a.source = A.v64.src[lv - 1].p;
            a.psi = A.v64.corr[lv - 1].p;
            a.pA = A.v64.cpA.p;
            a.wA = A.v64.cwA.p;
            a.rA = A.v64.crA.p;
            a.rD = A.v64.crD.p;
            a.maxIter = 1000;
            a.log = nullptr;
            a.logCount = A.coarseCount.p;
            a.logCapacity = 0;
            a.out = nullptr;
            args.push_back(a);
        }
        buildTiles(coarsestTiles, co, stream);
        maxTiles = std::max(maxTiles, coarsestTiles.nTiles);
        coarsestArgs.upload(args.data(), args.size(), stream);
    }
    // the batched sweep's shared-memory ceiling (this translation unit's instances)
    B2G_CUDA(cudaFuncSetAttribute(k::gsSweepBatch<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    B2G_CUDA(cudaFuncSetAttribute(k::gsSweepBatch<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    B2G_CUDA(cudaFuncSetAttribute(k::coarseDenseSolveBatch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(sizeof(double)) * k::kDenseMax * k::kDenseMax));
    partial.alloc(2 * static_cast<size_t>(maxTiles), stream);
    partial32.alloc(2 * static_cast<size_t>(maxTiles), stream);
    sf64.alloc(K, stream);
    sf32.alloc(K, stream);
    active.alloc(K, stream);
    active.zero(stream);
    nActive.alloc(1, stream);
    perf.alloc(K, stream);
    B2G_CUDA(cudaStreamSynchronize(stream));
}

// Each case's dense coarsest factor for its current coefficients, and the batched solve's table (the
// FP32 coarsest vectors of every case that has its factor, n = 0 for the others): a case is solved
// as it is alone, by its factor where it has one and by PCG-DIC where it has none.
void Batch::prepareDense()
{
    const int K = static_cast<int>(cases.size());
    std::vector<k::DenseCase> h(K, k::DenseCase{0, nullptr, nullptr, nullptr});
    int with = 0;
    for (int c = 0; c < K; ++c)
    {
        Matrix& A = *cases[c];
        A.ensureDense();
        const int lv = A.nLevels();
        if (!A.denseUse || lv == 0) continue;
        h[c].n = A.n(lv);
        h[c].L = A.denseL.p;
        h[c].b = A.v32.src[lv - 1].p;
        h[c].x = A.v32.corr[lv - 1].p;
        ++with;
    }
    // the factors were made on the cases' own streams
    for (Matrix* A : cases) B2G_CUDA(cudaStreamSynchronize(A->stream));
    denseAny = with > 0;
    denseAll = with == K;
    if (denseAny)
    {
        // refilled in place: a captured iteration graph names the table's address
        denseCases.ensure(h.size(), stream);
        B2G_CUDA(cudaMemcpyAsync(denseCases.p, h.data(), sizeof(k::DenseCase) * h.size(), cudaMemcpyHostToDevice,
                                 stream));
    }
    B2G_CUDA(cudaStreamSynchronize(stream));
}

// A hash of every device address the batch's iteration hands its kernels (its tables, the cases'
// buffers): a captured graph is replayed only while it is unchanged.
unsigned long long Batch::layoutFingerprint() const
{
    unsigned long long h = 1469598103934665603ull;
    auto mix = [&](const void* p) {
        h ^= reinterpret_cast<unsigned long long>(p);
        h *= 1099511628211ull;
    };
    for (const void* p : {(const void*)segD.p, (const void*)segF.p, (const void*)coarsestArgs.p,
                          (const void*)denseCases.p, (const void*)active.p, (const void*)nActive.p, (const void*)err.p,
                          (const void*)partial.p, (const void*)sf64.p, (const void*)partial32.p, (const void*)sf32.p,
                          (const void*)perf.p, (const void*)coarsestTiles.tiles.p})
        mix(p);
    for (const BatchLevel& B : lev)
    {
        for (const TileList* L : {&B.all, &B.up, &B.scale, &B.down})
        {
            mix(L->tiles.p);
            mix(L->segOf.p);
            mix(L->tileStart.p);
        }
        for (const void* p : {(const void*)B.gs64.p, (const void*)B.gs32.p, (const void*)B.parts.p,
                              (const void*)B.progress.p, (const void*)B.mcSmall.p})
            mix(p);
        for (const auto& kv : B.pipe)
        {
            mix(kv.second.table.p);
            mix(kv.second.caseOf.p);
            mix(kv.second.partsBig.p);
        }
        for (const TileList& L : B.mc) mix(L.tiles.p);
    }
    for (const Matrix* A : cases) h ^= A->layoutFingerprint() + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    return h;
}

// The multicolour layout of every case's levels (built on each mesh once) in the FP32 descriptors,
// and per level and colour the tiles of the swept cases' rows of that colour.
void Batch::prepareMulticolour()
{
    if (mcReady) return;
    const int K = static_cast<int>(cases.size());
    for (Matrix* A : cases)
    {
        A->ensureMulticolour();
        B2G_CUDA(cudaStreamSynchronize(A->stream));
    }
    for (int c = 0; c < K; ++c)
        for (int lv = 0; lv <= nLevelsOf[c]; ++lv)
        {
            const Colouring& C = cases[c]->mesh->lev[lv].mc;
            SegLevel<float>& f = hostF[segOfCase[c][lv]];
            f.mcPos = C.pos.p;
            f.mcSlice = C.sliceBase.p;
            f.mcCol = C.col.p;
            f.mcVal = cases[c]->v32.coef[lv].mcVal.p;
            f.mcDiag = cases[c]->v32.coef[lv].mcDiag.p;
            f.mcColourStart = C.colourStartD.p;
            f.mcColours = C.nColours;
            f.mcRows = C.nRows;
        }
    segF.upload(hostF.data(), hostF.size(), stream);
    // the batch's own autotuner: per level, the largest case that one block sweeps whole (one launch
    // for all of them) while the larger ones go by tiles, one launch per colour; every candidate is
    // timed on the level's own data and the fastest kept
    multicolour = true;
    B2G_CUDA(cudaMemsetAsync(active.p, 0xff, sizeof(int) * K, stream));  // every case swept while timing
    cudaEvent_t e0, e1;
    B2G_CUDA(cudaEventCreate(&e0));
    B2G_CUDA(cudaEventCreate(&e1));
    const long long l0 = launches;
    mcThreshold.assign(maxLevels + 1, 0);
    mcSweepMs.assign(maxLevels + 1, 0.f);
    for (int lv = 0; lv <= maxLevels; ++lv)
    {
        if (lev[lv].nParts == 0) continue;
        float best = 0.f;
        int bestThr = -1;
        for (int thr : {0, 4096, 16384, k::kMcSmallRows})
        {
            buildMcLists(lv, thr);
            smooth<float>(lv, 1);  // warm
            B2G_CUDA(cudaEventRecord(e0, stream));
            smooth<float>(lv, 2);
            B2G_CUDA(cudaEventRecord(e1, stream));
            B2G_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            B2G_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (bestThr < 0 || ms < best)
            {
                best = ms;
                bestThr = thr;
            }
        }
        buildMcLists(lv, bestThr);
        mcThreshold[lv] = bestThr;
        mcSweepMs[lv] = best / 2.f;
    }
    launches = l0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B2G_CUDA(cudaStreamSynchronize(stream));
    mcReady = true;
}

// The multicolour launch lists of level lv: cases with at most `threshold` rows are swept whole by
// one block each (one launch for all), the others by tiles of their rows, one launch per colour.
void Batch::buildMcLists(int lv, int threshold)
{
    const int K = static_cast<int>(cases.size());
    std::vector<int> small;
    auto isSmall = [&](int c) { return cases[c]->mesh->lev[lv].mc.nRows <= threshold; };
    int nCol = 0;
    for (int c = 0; c < K; ++c)
    {
        if (nLevelsOf[c] < lv + 1) continue;
        if (isSmall(c)) small.push_back(segOfCase[c][lv]);
        else nCol = std::max(nCol, cases[c]->mesh->lev[lv].mc.nColours);
    }
    lev[lv].nMcSmall = static_cast<int>(small.size());
    if (!small.empty()) lev[lv].mcSmall.upload(small.data(), small.size(), stream);
    lev[lv].mc.clear();
    lev[lv].mc.resize(nCol);
    for (int k = 0; k < nCol; ++k)
    {
        std::vector<int4> tiles;
        for (int c = 0; c < K; ++c)
        {
            if (nLevelsOf[c] < lv + 1 || isSmall(c)) continue;
            const Colouring& C = cases[c]->mesh->lev[lv].mc;
            if (k >= C.nColours) continue;
            const int sg = segOfCase[c][lv];
            for (int b = C.colourStart[k]; b < C.colourStart[k + 1]; b += kTile)
                tiles.push_back(make_int4(sg, b, std::min(C.colourStart[k + 1], b + kTile), 0));
        }
        TileList& L = lev[lv].mc[k];
        L.nTiles = static_cast<int>(tiles.size());
        if (!tiles.empty()) L.tiles.upload(tiles.data(), tiles.size(), stream);
    }
}

Batch::~Batch()
{
    if (graph.exec) cudaGraphExecDestroy(graph.exec);
    cudaStreamSynchronize(stream);
}

#define B2G_TILES(L) (L).nTiles, BT, 0, stream
#define B2G_WARPS(L) warpGrid((L).nSeg), BT, 0, stream

template <class T>
void Batch::smooth(int lv, int nSweeps)
{
    BatchLevel& B = lev[lv];
    if (nSweeps <= 0 || B.nParts == 0) return;
    if (sizeof(T) == 4 && multicolour)
    {
        const int rpsi = lv == 0 ? V_W : V_CORR;
        const int rsrc = lv == 0 ? V_R : V_SRC;
        if (B.nMcSmall)
        {
            bMcSmoothSmall<<<B.nMcSmall, 1024, 0, stream>>>(B.mcSmall.p, segF.p, rpsi, rsrc, nSweeps, active.p);
            ++launches;
        }
        for (int sw = 0; sw < nSweeps; ++sw)
            for (const TileList& L : B.mc)
            {
                if (L.nTiles == 0) continue;
                bMcSweep<<<L.nTiles, BT, 0, stream>>>(L.tiles.p, segF.p, rpsi, rsrc, active.p);
                ++launches;
            }
        B2G_LAUNCH_CHECK();
        return;
    }
    const k::GsArgs<T>* args = sizeof(T) == 8 ? reinterpret_cast<const k::GsArgs<T>*>(B.gs64.p)
                                              : reinterpret_cast<const k::GsArgs<T>*>(B.gs32.p);
    const size_t smem = sizeof(T) == 8 ? B.smem64 : B.smem32;
    const int4* parts = B.parts.p;
    int nParts = B.nParts;
    auto pit = B.pipe.find(nSweeps * 16 + static_cast<int>(sizeof(T)));
    if (pipeOn && pit != B.pipe.end() && pit->second.use)
    {
        // the cases whose level fits one CTA: every sweep in one pipelined launch; the rest below
        const BatchLevel::Pipe& P = pit->second;
        if (P.nSmall)
        {
            launchPipeBatch<T>(P.table.p, P.caseOf.p, P.nSmall, P.smem, active.p, stream);
            ++launches;
        }
        parts = P.partsBig.p;
        nParts = P.nPartsBig;
    }
    if (nParts == 0) return;
    for (int sw = 0; sw < nSweeps; ++sw)
    {
        B2G_CUDA(cudaMemsetAsync(B.progress.p, 0, B.progress.bytes(), stream));
        k::gsSweepBatch<T><<<nParts, B.block, smem, stream>>>(
            args, parts, active.p, reinterpret_cast<int*>(B.progress.p + B.ticketAt));
        B2G_LAUNCH_CHECK();
        ++launches;
    }
}

// The batched pipelined sweeps of level lv for nSweeps sweeps in T: per case whose level fits one
// CTA's shared memory, the one-CTA schedule (on its mesh, built once) with that case's vectors; the
// other cases' parts for the sweep-by-sweep launch. Outside any capture.
template <class T>
void Batch::preparePipe(int lv, int nSweeps)
{
    BatchLevel& B = lev[lv];
    const int key = nSweeps * 16 + static_cast<int>(sizeof(T));
    if (B.nParts == 0) return;
    if (B.pipe.count(key)) return;
    BatchLevel::Pipe& P = B.pipe[key];
    const int K = static_cast<int>(cases.size());
    std::vector<k::PipeArgs<T>> table;
    std::vector<int> caseOf;
    std::vector<char> small(K, 0);
    for (int c = 0; c < K; ++c)
    {
        if (nLevelsOf[c] < lv + 1 || lv > nLevelsOf[c]) continue;
        Matrix& A = *cases[c];
        LevelAddr& L = A.mesh->lev[lv];
        if (L.nCells == 0) continue;
        const PipeSchedule* S = pipeOneCta(L, nSweeps, sizeof(T), stream);
        if (!S) continue;
        const T* b;
        T* psi;
        if (sizeof(T) == 8)
        {
            b = reinterpret_cast<const T*>(lv == 0 ? A.rA.p : A.v64.src[lv - 1].p);
            psi = reinterpret_cast<T*>(lv == 0 ? A.wA.p : A.v64.corr[lv - 1].p);
        }
        else
        {
            b = reinterpret_cast<const T*>(lv == 0 ? A.r32.p : A.v32.src[lv - 1].p);
            psi = reinterpret_cast<T*>(lv == 0 ? A.w32.p : A.v32.corr[lv - 1].p);
        }
        table.push_back(A.pipeArgs<T>(lv, *S, psi, b));
        caseOf.push_back(c);
        small[c] = 1;
        P.smem = std::max(P.smem, pipeSmemBytes(*S, sizeof(T)));
    }
    std::vector<int4> big;
    for (const int4& q : B.hostParts)
        if (!small[q.z]) big.push_back(q);
    P.nSmall = static_cast<int>(table.size());
    P.nPartsBig = static_cast<int>(big.size());
    if (P.nSmall)
    {
        P.table.upload(reinterpret_cast<const unsigned char*>(table.data()), sizeof(k::PipeArgs<T>) * table.size(),
                       stream);
        P.caseOf.upload(caseOf.data(), caseOf.size(), stream);
    }
    if (P.nPartsBig) P.partsBig.upload(big.data(), big.size(), stream);
    B2G_CUDA(cudaStreamSynchronize(stream));
    if (!P.nSmall) return;
    // the batch's own choice, by measurement: the pipelined launch for the small cases' levels, or the
    // sweep-by-sweep launches for every case (the same bits either way); every case swept while timing
    B2G_CUDA(cudaMemsetAsync(active.p, 0xff, sizeof(int) * K, stream));
    cudaEvent_t e0, e1;
    B2G_CUDA(cudaEventCreate(&e0));
    B2G_CUDA(cudaEventCreate(&e1));
    const long long l0 = launches;
    auto timeIt = [&](bool use) {
        P.use = use;
        smooth<T>(lv, nSweeps);  // warm
        B2G_CUDA(cudaEventRecord(e0, stream));
        for (int i = 0; i < 2; ++i) smooth<T>(lv, nSweeps);
        B2G_CUDA(cudaEventRecord(e1, stream));
        B2G_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        B2G_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 2.f;
    };
    P.msPipe = timeIt(true);
    P.msSweeps = timeIt(false);
    P.use = P.msPipe < P.msSweeps;
    launches = l0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Every batched pipelined sweep the controls' V-cycle makes, before the iterations run.
void Batch::preparePipes(const b2g_controls& c)
{
    pipeOn = g_pipeline && !multicolour && c.smoother == B2G_SMOOTHER_GAUSS_SEIDEL;
    if (!pipeOn) return;
    const bool fp64 = c.precision == B2G_PRECISION_FP64;
    auto want = [&](int lv, int s) {
        if (s <= 0 || lv >= static_cast<int>(lev.size())) return;
        if (fp64) preparePipe<double>(lv, s);
        else preparePipe<float>(lv, s);
    };
    want(0, c.nFinestSweeps);
    for (int lv = 1; lv < static_cast<int>(lev.size()); ++lv)
    {
        const int li = lv - 1;
        want(lv, std::min(c.nPostSweeps + c.postSweepsLevelMultiplier * li, c.maxPostSweeps));
        if (c.nPreSweeps) want(lv, std::min(c.nPreSweeps + c.preSweepsLevelMultiplier * li, c.maxPreSweeps));
    }
}

template <class T>
void Batch::scale(int lv, const TileList& L, int field, int acf, int src, bool finest, int psiRole)
{
    if (L.nTiles == 0) return;
    SegLevel<T>* S = segs<T>();
    T* sf = sizeof(T) == 8 ? reinterpret_cast<T*>(sf64.p) : reinterpret_cast<T*>(sf32.p);
    T* part = sizeof(T) == 8 ? reinterpret_cast<T*>(partial.p) : reinterpret_cast<T*>(partial32.p);
    (void)lv;
    if (serial && sizeof(T) == 8)
    {
        bAmul<T><<<B2G_TILES(L)>>>(L.tiles.p, S, field, acf, active.p);
        bSerialScaleDots<<<B2G_WARPS(L)>>>(L.segOf.p, L.nSeg, segD.p, field, src, acf, sf64.p, active.p);
    }
    else
    {
        bAmulScaleDots<T><<<B2G_TILES(L)>>>(L.tiles.p, S, field, src, acf, part, active.p);
        bScaleFactor<T><<<B2G_WARPS(L)>>>(L.segOf.p, L.tileStart.p, L.nSeg, S, part, sf, active.p);
    }
    if (finest)
        bScaleUpdateAdd<T><<<B2G_TILES(L)>>>(L.tiles.p, S, sf, field, src, acf, psiRole, active.p);
    else
        bScaleUpdate<T><<<B2G_TILES(L)>>>(L.tiles.p, S, sf, field, src, acf, active.p);
    B2G_LAUNCH_CHECK();
    launches += 3;
}

// GAMGSolver::Vcycle (GAMG:627-735) for every case at once: psi = V_W, source = V_R, Apsi = V_AWA,
// the finest correction V_FC, the residual `fresRole` (V_R, or V_FR between V-cycles)
template <class T>
void Batch::vcycle(const b2g_controls& c, int fresRole)
{
    SegLevel<T>* S = segs<T>();
    const int* act = active.p;
    // down: restrict level 0, then pre-smooth (optional) and restrict every coarse level
    if (lev[0].down.nTiles) bRestrict<T><<<B2G_TILES(lev[0].down)>>>(lev[0].down.tiles.p, S, fresRole, V_SRC, act);
    ++launches;
    for (int lv = 1; lv < maxLevels; ++lv)
    {
        BatchLevel& B = lev[lv];
        if (B.up.nTiles == 0) continue;
        const int li = lv - 1;
        if (c.nPreSweeps)
        {
            bZero<T><<<B2G_TILES(B.up)>>>(B.up.tiles.p, S, V_CORR, act);
            smooth<T>(lv, std::min(c.nPreSweeps + c.preSweepsLevelMultiplier * li, c.maxPreSweeps));
            if (c.scaleCorrection) scale<T>(lv, B.scale, V_CORR, V_ACF, V_SRC, false, -1);
            bResidual<T><<<B2G_TILES(B.up)>>>(B.up.tiles.p, S, V_SRC, V_CORR, V_SRC, act);
            launches += 2;
        }
        bRestrict<T><<<B2G_TILES(B.down)>>>(B.down.tiles.p, S, V_SRC, V_SRC, act);
        ++launches;
    }
    B2G_LAUNCH_CHECK();
    // each case's coarsest level: PCG-DIC from zero, in FP64 (the FP32 form widens and narrows)
    bZero<T><<<B2G_TILES(coarsestTiles)>>>(coarsestTiles.tiles.p, S, V_CORR, act);
    const int K = static_cast<int>(cases.size());
    if (sizeof(T) == 8)
    {
        k::coarsestPcgDicBatch<<<K, 32, 0, stream>>>(coarsestArgs.p, c.precTolerance, c.precRelTol, act);
        launches += 2;
    }
    else
    {
        // the FP32 forms: PCG-DIC in FP64 for the cases without a dense factor (for every active case,
        // unless all have one), then the cases' dense Cholesky factors, one warp each, whose solves
        // overwrite the corrections of the cases that have one
        if (!(denseNow && denseAll))
        {
            bCast<double, float><<<B2G_TILES(coarsestTiles)>>>(coarsestTiles.tiles.p, segD.p, segF.p, V_SRC, V_SRC, act);
            bCast<double, float><<<B2G_TILES(coarsestTiles)>>>(coarsestTiles.tiles.p, segD.p, segF.p, V_CORR, V_CORR, act);
            // the single-case FP32 form hands the FP64 solve tolerances rounded to float
            k::coarsestPcgDicBatch<<<K, 32, 0, stream>>>(coarsestArgs.p, static_cast<double>(static_cast<float>(c.precTolerance)),
                                                         static_cast<double>(static_cast<float>(c.precRelTol)), act);
            bCast<float, double><<<B2G_TILES(coarsestTiles)>>>(coarsestTiles.tiles.p, segF.p, segD.p, V_CORR, V_CORR, act);
            launches += 5;
        }
        if (denseNow)
        {
            k::coarseDenseSolveBatch<<<K, 32, sizeof(double) * k::kDenseMax * k::kDenseMax, stream>>>(denseCases.p,
                                                                                                    act);
            ++launches;
        }
    }
    B2G_LAUNCH_CHECK();
    // up
    for (int lv = maxLevels - 1; lv >= 1; --lv)
    {
        BatchLevel& B = lev[lv];
        if (B.up.nTiles == 0) continue;
        const int li = lv - 1;
        if (c.nPreSweeps) bCopy<T><<<B2G_TILES(B.up)>>>(B.up.tiles.p, S, V_PRE, V_CORR, act);
        bProlong<T><<<B2G_TILES(B.up)>>>(B.up.tiles.p, S, V_CORR, V_CORR, act);
        ++launches;
        if (c.scaleCorrection) scale<T>(lv, B.scale, V_CORR, V_ACF, V_SRC, false, -1);
        if (c.nPreSweeps)
        {
            bAdd<T><<<B2G_TILES(B.up)>>>(B.up.tiles.p, S, V_CORR, V_PRE, act);
            launches += 2;
        }
        B2G_LAUNCH_CHECK();
        smooth<T>(lv, std::min(c.nPostSweeps + c.postSweepsLevelMultiplier * li, c.maxPostSweeps));
    }
    // finest
    BatchLevel& F = lev[0];
    bProlong<T><<<B2G_TILES(F.all)>>>(F.all.tiles.p, S, V_CORR, V_FC, act);
    ++launches;
    if (c.scaleCorrection) scale<T>(0, F.all, V_FC, V_AWA, fresRole, true, V_W);
    else
    {
        bAdd<T><<<B2G_TILES(F.all)>>>(F.all.tiles.p, S, V_W, V_FC, act);
        ++launches;
    }
    B2G_LAUNCH_CHECK();
    smooth<T>(0, c.nFinestSweeps);
}

// GAMGPreconditioner::precondition (GAMG:1089-1107): W from R on every active case
void Batch::precondition(const b2g_controls& c)
{
    const TileList& L = lev[0].all;
    const int* act = active.p;
    if (c.precision != B2G_PRECISION_FP64)
    {
        bCast<float, double><<<B2G_TILES(L)>>>(L.tiles.p, segF.p, segD.p, V_R, V_R, act);
        bZero<float><<<B2G_TILES(L)>>>(L.tiles.p, segF.p, V_W, act);
        launches += 2;
        int fres = V_R;
        for (int cycle = 0; cycle < c.nVcycles; ++cycle)
        {
            vcycle<float>(c, fres);
            if (cycle < c.nVcycles - 1)
            {
                bAmul<float><<<B2G_TILES(L)>>>(L.tiles.p, segF.p, V_W, V_AWA, act);
                bSubtract<float><<<B2G_TILES(L)>>>(L.tiles.p, segF.p, V_R, V_AWA, V_FR, act);
                launches += 2;
                fres = V_FR;
            }
        }
        bCast<double, float><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, segF.p, V_W, V_W, act);
        ++launches;
        B2G_LAUNCH_CHECK();
        return;
    }
    bZero<double><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_W, act);
    ++launches;
    int fres = V_R;
    for (int cycle = 0; cycle < c.nVcycles; ++cycle)
    {
        vcycle<double>(c, fres);
        if (cycle < c.nVcycles - 1)
        {
            bAmul<double><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_W, V_AWA, act);
            bSubtract<double><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_R, V_AWA, V_FR, act);
            launches += 2;
            fres = V_FR;
        }
    }
    B2G_LAUNCH_CHECK();
}

// a sum over every active case's finest cells into its scalars at byte offset `off`
void Batch::reduce(int op, int a, int b, size_t off)
{
    const TileList& L = lev[0].all;
    const int* act = active.p;
    if (serial)
    {
        if (op == k::RED_DOT) bSerialReduce<k::RED_DOT><<<B2G_WARPS(L)>>>(L.segOf.p, L.nSeg, segD.p, a, b, off, act);
        else if (op == k::RED_SUMMAG)
            bSerialReduce<k::RED_SUMMAG><<<B2G_WARPS(L)>>>(L.segOf.p, L.nSeg, segD.p, a, b, off, act);
        else bSerialReduce<k::RED_SUM><<<B2G_WARPS(L)>>>(L.segOf.p, L.nSeg, segD.p, a, b, off, act);
        ++launches;
    }
    else
    {
        if (op == k::RED_DOT) bReducePartial<k::RED_DOT><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, a, b, partial.p, act);
        else if (op == k::RED_SUMMAG)
            bReducePartial<k::RED_SUMMAG><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, a, b, partial.p, act);
        else bReducePartial<k::RED_SUM><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, a, b, partial.p, act);
        bReduceFinal<<<B2G_WARPS(L)>>>(L.segOf.p, L.tileStart.p, L.nSeg, segD.p, partial.p, off, act);
        launches += 2;
    }
    B2G_LAUNCH_CHECK();
}

// one PCG iteration of every active case (the body of PCG.C's loop), then who goes on
void Batch::iteration(const b2g_controls& c)
{
    const TileList& L = lev[0].all;
    const int* act = active.p;
    const bool flexible = c.precision != B2G_PRECISION_FP64;
    const int K = static_cast<int>(cases.size());
    precondition(c);
    reduce(k::RED_DOT, V_W, V_R, offsetof(PcgScalars, wArA));
    if (flexible) reduce(k::RED_DOT, V_W, V_ROLD, offsetof(PcgScalars, wrOld));
    bPUpdate<<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_W, V_P, flexible ? 1 : 0, act);
    bAmul<double><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_P, V_W, act);
    launches += 2;
    reduce(k::RED_DOT, V_W, V_P, offsetof(PcgScalars, wApA));
    bAlphaUpdate<<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_PSI, V_P, V_R, V_W, flexible ? V_ROLD : -1, partial.p, act);
    ++launches;
    if (serial) reduce(k::RED_SUMMAG, V_R, -1, offsetof(PcgScalars, sumMag));
    else
    {
        bReduceFinal<<<B2G_WARPS(L)>>>(L.segOf.p, L.tileStart.p, L.nSeg, segD.p, partial.p,
                                       offsetof(PcgScalars, sumMag), act);
        ++launches;
    }
    B2G_CUDA(cudaMemsetAsync(nActive.p, 0, sizeof(int), stream));
    bFinish<<<ceilDiv(K, 128), 128, 0, stream>>>(K, segD.p, c.tolerance, c.relTol, c.maxIter, c.minIter, active.p,
                                                 nActive.p);
    ++launches;
    B2G_LAUNCH_CHECK();
}

void Batch::solve(const b2g_controls& c, const double* const* source, double* const* psi, int memspace,
                  b2g_perf* perfs)
{
    if (c.solver != B2G_SOLVER_PCG_GAMG)
        fail(B2G_ERR_REFUSED, "b2g batch: the batched solve is PCG with the GAMG preconditioner.");
    if (c.smoother != B2G_SMOOTHER_GAUSS_SEIDEL)
        fail(B2G_ERR_REFUSED, "b2g: the device smoother for this entry is GaussSeidel only so far; "
                              "symGaussSeidel, DIC and DICGaussSeidel are not built on the device yet.");
    if (memspace != B2G_MEM_HOST && memspace != B2G_MEM_DEVICE) fail(B2G_ERR_ARGUMENT, "b2g batch: bad memspace");
    if (c.precision < B2G_PRECISION_FP64 || c.precision > B2G_PRECISION_FP32_PRECOND_MULTICOLOUR)
        fail(B2G_ERR_ARGUMENT, "b2g batch: unknown precision form");
    multicolour = c.precision == B2G_PRECISION_FP32_PRECOND_MULTICOLOUR;
    if (multicolour) prepareMulticolour();
    denseNow = false;
    if (c.precision != B2G_PRECISION_FP64 && c.coarsestDirect)
    {
        prepareDense();
        denseNow = denseAny;
    }
    preparePipes(c);
    const int K = static_cast<int>(cases.size());
    serial = c.reduction == B2G_REDUCTION_SERIAL;
    launches = 0;
    const cudaMemcpyKind in = memspace == B2G_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out = memspace == B2G_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < K; ++k)
    {
        const size_t bytes = sizeof(double) * cases[k]->n(0);
        if (!source[k] || !psi[k]) fail(B2G_ERR_ARGUMENT, "b2g batch: null field");
        B2G_CUDA(cudaMemcpyAsync(cases[k]->fc.p, source[k], bytes, in, stream));
        B2G_CUDA(cudaMemcpyAsync(cases[k]->fr.p, psi[k], bytes, in, stream));
    }
    const TileList& L = lev[0].all;
    bPermute<<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_FC, V_SOURCE, 1);
    bPermute<<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_FR, V_PSI, 1);
    bAmul<double><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_PSI, V_W, nullptr);
    bSubtract<double><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_SOURCE, V_W, V_R, nullptr);
    launches += 4;
    // normFactor (GAMG:119-159)
    if (serial)
    {
        bSerialNormFactor<<<B2G_WARPS(L)>>>(L.segOf.p, L.nSeg, segD.p, V_PSI, V_SOURCE, V_W);
        ++launches;
    }
    else
    {
        bReducePartial<k::RED_SUM><<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_PSI, -1, partial.p, nullptr);
        bReduceFinal<<<B2G_WARPS(L)>>>(L.segOf.p, L.tileStart.p, L.nSeg, segD.p, partial.p,
                                       offsetof(PcgScalars, sumPsi), nullptr);
        bNormFactorPartial<<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_PSI, V_SOURCE, V_W, partial.p);
        bReduceFinal<<<B2G_WARPS(L)>>>(L.segOf.p, L.tileStart.p, L.nSeg, segD.p, partial.p,
                                       offsetof(PcgScalars, nf), nullptr);
        bNfFinish<<<ceilDiv(K, 128), 128, 0, stream>>>(K, segD.p);
        launches += 5;
    }
    B2G_LAUNCH_CHECK();
    // the initial residual's sum of magnitudes, with every case counted
    B2G_CUDA(cudaMemsetAsync(active.p, 0xff, sizeof(int) * K, stream));  // nonzero: every case
    reduce(k::RED_SUMMAG, V_R, -1, offsetof(PcgScalars, sumMag));
    B2G_CUDA(cudaMemsetAsync(nActive.p, 0, sizeof(int), stream));
    bStart<<<ceilDiv(K, 128), 128, 0, stream>>>(K, segD.p, c.tolerance, c.relTol, c.minIter, active.p, nActive.p);
    ++launches;
    B2G_LAUNCH_CHECK();
    int going = 0;
    B2G_CUDA(cudaMemcpyAsync(&going, nActive.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    while (going > 0)
    {
        // one captured graph per controls and reduction order
        std::vector<unsigned char> key(sizeof(b2g_controls) + 1 + sizeof(unsigned long long));
        std::memcpy(key.data(), &c, sizeof(b2g_controls));
        key[sizeof(b2g_controls)] = static_cast<unsigned char>((serial ? 1 : 0) | (denseNow ? 2 : 0) | (pipeOn ? 4 : 0) |
                                                               (denseAll ? 8 : 0) | (multicolour ? 16 : 0));
        const unsigned long long fp = layoutFingerprint();
        std::memcpy(key.data() + sizeof(b2g_controls) + 1, &fp, sizeof(fp));
        if (eagerIterations == 0 && (!graph.exec || graph.key != key))
        {
            // a batch's first iteration runs as plain launches: capturing pays off only from the
            // first replay, and many batches (a serving group) iterate once
            ++eagerIterations;
            iteration(c);
        }
        else if (!graph.exec || graph.key != key)
        {
            if (graph.exec) B2G_CUDA(cudaGraphExecDestroy(graph.exec));
            graph.exec = nullptr;
            const long long l0 = launches;
            B2G_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try
            {
                iteration(c);
            }
            catch (...)
            {
                cudaGraph_t dropped = nullptr;
                cudaStreamEndCapture(stream, &dropped);
                if (dropped) cudaGraphDestroy(dropped);
                throw;
            }
            cudaGraph_t g = nullptr;
            B2G_CUDA(cudaStreamEndCapture(stream, &g));
            const cudaError_t e = cudaGraphInstantiate(&graph.exec, g, 0);
            cudaGraphDestroy(g);
            B2G_CUDA(e);
            graph.launchesPerReplay = launches - l0;
            graph.key = std::move(key);
        }
        else
        {
            launches += graph.launchesPerReplay;
        }
        if (graph.exec && graph.key == key) B2G_CUDA(cudaGraphLaunch(graph.exec, stream));
        B2G_CUDA(cudaMemcpyAsync(&going, nActive.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
        B2G_CUDA(cudaStreamSynchronize(stream));
    }
    bPermute<<<B2G_TILES(L)>>>(L.tiles.p, segD.p, V_PSI, V_FC, 0);
    bGatherPerf<<<ceilDiv(K, 128), 128, 0, stream>>>(K, segD.p, perf.p);
    launches += 2;
    B2G_LAUNCH_CHECK();
    for (int k = 0; k < K; ++k)
        B2G_CUDA(cudaMemcpyAsync(psi[k], cases[k]->fc.p, sizeof(double) * cases[k]->n(0), out, stream));
    std::vector<BatchPerf> hp(K);
    B2G_CUDA(cudaMemcpyAsync(hp.data(), perf.p, sizeof(BatchPerf) * K, cudaMemcpyDeviceToHost, stream));
    int e = 0;
    B2G_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    if (e)
    {
        err.zero(stream);
        fail(B2G_ERR_DEVICE_TIMEOUT,
             "b2g: a bounded device-side wait in the Gauss-Seidel sweep gave up; the result is invalid.");
    }
    for (int k = 0; k < K; ++k)
    {
        perfs[k].initialResidual = hp[k].initialResidual;
        perfs[k].finalResidual = hp[k].finalResidual;
        perfs[k].nIterations = hp[k].nIterations;
    }
}

}  // namespace b2g

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------

namespace {

// Batch streams are never destroyed. A batch builds layouts that its meshes keep (the one-CTA
// pipelined schedules of pipeOneCta) on its own stream, and a mesh frees them on that stream when it
// goes, which may be long after the batch: a destroyed batch hands its stream back here, idle, for
// the next batch on the same device.
std::mutex g_batchStreamMu;
std::vector<std::pair<int, cudaStream_t>> g_idleBatchStreams;  // (device, stream)

cudaStream_t takeBatchStream(int device)
{
    {
        std::lock_guard<std::mutex> lk(g_batchStreamMu);
        for (size_t i = 0; i < g_idleBatchStreams.size(); ++i)
            if (g_idleBatchStreams[i].first == device)
            {
                const cudaStream_t s = g_idleBatchStreams[i].second;
                g_idleBatchStreams.erase(g_idleBatchStreams.begin() + static_cast<std::ptrdiff_t>(i));
                return s;
            }
    }
    cudaStream_t s = nullptr;
    B2G_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

void giveBackBatchStream(int device, cudaStream_t s)
{
    cudaStreamSynchronize(s);
    std::lock_guard<std::mutex> lk(g_batchStreamMu);
    g_idleBatchStreams.emplace_back(device, s);
}

}  // namespace

struct b2g_batch
{
    int device = 0;
    cudaStream_t stream = nullptr;
    std::unique_ptr<b2g::Batch> batch;
    ~b2g_batch()
    {
        batch.reset();
        if (stream) giveBackBatchStream(device, stream);
    }
};

using b2g::capi::guarded;
using b2g::capi::need;

extern "C" {

B2G_API b2g_status b2g_batch_create(b2g_matrix* const* matrices, int count, b2g_batch** out)
{
    return guarded([&] {
        need(out != nullptr, "b2g_batch_create: null output handle");
        *out = nullptr;
        need(matrices != nullptr && count >= 1, "b2g_batch_create: no matrices");
        std::vector<b2g::Matrix*> cs;
        for (int i = 0; i < count; ++i)
        {
            need(matrices[i] != nullptr && matrices[i]->mat, "b2g_batch_create: null matrix");
            cs.push_back(matrices[i]->mat.get());
        }
        std::unique_ptr<b2g_batch> h(new b2g_batch);
        B2G_CUDA(cudaGetDevice(&h->device));
        h->stream = takeBatchStream(h->device);
        h->batch.reset(new b2g::Batch(std::move(cs), h->stream));
        *out = h.release();
    });
}

B2G_API b2g_status b2g_batch_solve(b2g_batch* b, const double* const* sources, double* const* psis,
                                   const b2g_controls* controls, int memspace, b2g_perf* perfs)
{
    return guarded([&] {
        need(b && sources && psis && controls && perfs, "b2g_batch_solve: null argument");
        b->batch->solve(*controls, sources, psis, memspace, perfs);
    });
}

B2G_API b2g_status b2g_batch_launches(const b2g_batch* b, long long* launches)
{
    return guarded([&] {
        need(b && launches, "b2g_batch_launches: null argument");
        *launches = b->batch->launches;
    });
}

B2G_API b2g_status b2g_batch_destroy(b2g_batch* b)
{
    return guarded([&] { delete b; });
}

}  // extern "C"
