// solver.cu -- the V-cycle, the PCG with the GAMG preconditioner and the standalone GAMG solver,
// orchestrated on one stream with every scalar kept on the device.
//
// Reference: GAMG = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu
#include "solver.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

namespace b2g {

bool g_profiling = false;
bool g_pipeline = true;
std::atomic<int> g_partCells{48};

namespace {

constexpr int NT = 256;          // threads of the row and reduction kernels
constexpr int kResidentMaxCells = 24576;         // the largest level the resident sweep takes
constexpr size_t kResidentSmem = 200 * 1024;     // its shared memory: psi of the level and the depth ranges
constexpr int kMaxPartials = 1024;

int rowsGrid(int n)
{
    const int g = ceilDiv(std::max(n, 1), NT);
    return std::min(g, 16 * DeviceInfo::get().numSMs);
}
int redGrid(int n) { return std::min(ceilDiv(std::max(n, 1), NT), kMaxPartials); }

constexpr double kSmall = 1e-20;   // GAMG:16
constexpr double kVSmall = 1e-300; // GAMG:17
constexpr double kGreat = 1e+20;   // GAMG:19

__global__ void kInitResidual(PcgScalars* s)
{
    s->initRes = s->sumMag / s->nf;
    s->finalRes = s->initRes;
}

__global__ void kNfFinish(PcgScalars* s)
{
    s->nf = __dadd_rn(s->nf, kSmall);
}

__global__ void kPcgStart(PcgScalars* s)
{
    s->wArA = kGreat;
    s->wArAold = kGreat;
    s->iter = 0;
    s->singular = 0;
}

// p = w (first iteration) or p = w + beta*p with beta = wArA/wArAold (PCG.C), or the flexible
// Polak-Ribiere+ beta of the FP32-preconditioned form, max(0, (z.r_new - z.r_old)/rho_old)
// (device_amg_pcg.cu:36-48)
__global__ void kPUpdate(int n, const double* __restrict__ w, double* __restrict__ p, const PcgScalars* s,
                         int flexible)
{
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
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        p[c] = iter == 0 ? w[c] : __dadd_rn(w[c], __dmul_rn(beta, p[c]));
    }
}

// checkSingularity, then psi += alpha*p, r -= alpha*w, with the partial sums of |r| (PCG.C)
template <int NTT>
__global__ void __launch_bounds__(NTT) kAlphaUpdate(int n, double* __restrict__ psi, const double* __restrict__ p,
                                                    double* __restrict__ r, const double* __restrict__ w,
                                                    double* __restrict__ rOld, PcgScalars* s,
                                                    double* __restrict__ partial)
{
    __shared__ double sh[NTT / 32];
    const double wApA = s->wApA;
    const bool singular = __ddiv_rn(fabs(wApA), s->nf) < kVSmall;
    if (singular)
    {
        if (blockIdx.x == 0 && threadIdx.x == 0) s->singular = 1;
        if (threadIdx.x == 0) partial[blockIdx.x] = 0.0;
        return;
    }
    const double alpha = __ddiv_rn(s->wArA, wApA);
    double acc = 0.0;
    for (int c = blockIdx.x * NTT + threadIdx.x; c < n; c += gridDim.x * NTT)
    {
        const double rc = r[c];
        if (rOld) rOld[c] = rc;
        psi[c] = __dadd_rn(psi[c], __dmul_rn(alpha, p[c]));
        const double rn = __dsub_rn(rc, __dmul_rn(alpha, w[c]));
        r[c] = rn;
        acc = __dadd_rn(acc, fabs(rn));
    }
    acc = k::blockSum<double, NTT>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void kIterFinish(PcgScalars* s)
{
    if (s->singular) return;
    s->finalRes = __ddiv_rn(s->sumMag, s->nf);
    s->wArAold = s->wArA;
    s->iter += 1;
}

__global__ void kResidualFinish(PcgScalars* s)
{
    s->finalRes = __ddiv_rn(s->sumMag, s->nf);
}

template <class T>
__global__ void kZero(long long n, T* x)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = T(0);
}

bool convergedH(double fin, double init, double tol, double relTol)
{
    return fin < tol || (relTol > kSmall && fin < relTol * init);
}


// the position-ordered coefficients of one level: diagonal and CSR rows
__global__ void kGsLayout(int n, long long nnz, const int* __restrict__ posCell, const int* __restrict__ entFacePos,
                          const double* __restrict__ diag, const double* __restrict__ upper, double* __restrict__ gsDiag,
                          double* __restrict__ rowVal)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long m = max(static_cast<long long>(n), nnz);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += stride)
    {
        if (i < n) gsDiag[i] = diag[posCell[i]];
        if (i < nnz) rowVal[i] = upper[entFacePos[i]];
    }
}

// (+8 elements of zeroed padding past the diagonal: bulk copies round position ranges out to 16 bytes)
// The padding of the diagonal and of the chunk blobs is zeroed when the buffers are new; a refill with
// new coefficients writes the same bytes as the first fill, so the padding stays zero.
template <class T>
void allocGsLayout(const LevelAddr& L, LevelCoef<T>& C, cudaStream_t s)
{
    const void* diagWas = C.gsDiag.p;
    const size_t diagN = C.gsDiag.n;
    C.gsDiag.ensure(L.nCells + 8, s);
    if (C.gsDiag.p != diagWas || C.gsDiag.n != diagN) C.gsDiag.zero(s);
    C.rowVal.ensure(std::max<size_t>(2 * (size_t)L.nFaces, 1), s);
    const long long bytes = sizeof(T) == 8 ? L.gs.blobBytes64 : L.gs.blobBytes32;
    const void* blobWas = C.blob.p;
    const size_t blobN = C.blob.n;
    C.blob.ensure(static_cast<size_t>(std::max<long long>(bytes, 16)), s);
    if (C.blob.p != blobWas || C.blob.n != blobN) C.blob.zero(s);
}

// the sweep's chunk blobs in T, from the FP64 LDU coefficients
template <class T>
void fillBlobs(const LevelAddr& L, LevelCoef<T>& C, const double* upper, cudaStream_t s)
{
    const GsSchedule& G = L.gs;
    if (G.nChunks)
        k::buildChunkBlobs<T><<<std::min(G.nChunks, 65535), 128, 0, s>>>(
            G.nChunks, reinterpret_cast<const int4*>(G.chunkRec.p), C.gsDiag.p, G.posEnt.p, G.gsCode.p,
            G.gsEntFace.p, upper, C.blob.p, nullptr);
    B2G_LAUNCH_CHECK();
}

// the level's sliced ELL coefficients from its CSR ones (GsSchedule::ellEnt), where it has the layout
template <class T>
__global__ void kEllValues(long long nEnt, const int* __restrict__ ellEnt, const T* __restrict__ rowVal,
                           T* __restrict__ ellVal)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nEnt; e += (long long)gridDim.x * blockDim.x)
    {
        const int q = ellEnt[e];
        ellVal[e] = q >= 0 ? rowVal[q] : T(0);
    }
}

template <class T>
void fillEll(const LevelAddr& L, LevelCoef<T>& C, cudaStream_t s)
{
    if (!L.gs.nEllEnt) return;
    C.ellVal.ensure(static_cast<size_t>(L.gs.nEllEnt), s);
    kEllValues<T><<<std::min(ceilDiv(L.gs.nEllEnt, NT), 8192), NT, 0, s>>>(L.gs.nEllEnt, L.gs.ellEnt.p, C.rowVal.p,
                                                                         C.ellVal.p);
    B2G_LAUNCH_CHECK();
}

void fillGsLayout(const LevelAddr& L, LevelCoef<double>& C, cudaStream_t s)
{
    allocGsLayout(L, C, s);
    const long long nnz = 2LL * L.nFaces;
    const long long m = std::max<long long>(L.nCells, nnz);
    if (m)
        kGsLayout<<<std::min(ceilDiv(m, NT), 8192), NT, 0, s>>>(L.nCells, nnz, L.gs.posCell.p, L.gs.entFacePos.p,
                                                                C.diag.p, C.upper.p, C.gsDiag.p, C.rowVal.p);
    B2G_LAUNCH_CHECK();
    fillEll<double>(L, C, s);
    fillBlobs<double>(L, C, C.upper.p, s);
}

template <class T, class S>
void castInto(long long n, const S* in, T* out, cudaStream_t s)
{
    if (n) k::castArray<T, S><<<std::min(ceilDiv(n, NT), 4096), NT, 0, s>>>(n, in, out);
    B2G_LAUNCH_CHECK();
}

template <class T>
void zeroArray(long long n, T* x, cudaStream_t s)
{
    if (n) kZero<T><<<std::min(ceilDiv(n, NT), 4096), NT, 0, s>>>(n, x);
    B2G_LAUNCH_CHECK();
}

}  // namespace

namespace k {

__global__ void mcSweep(int rowBegin, int rowEnd, const int* __restrict__ pos, const int* __restrict__ sliceBase,
                        const int* __restrict__ col, const float* __restrict__ val, const float* __restrict__ diag,
                        const float* __restrict__ b, float* __restrict__ psi)
{
    for (int r = rowBegin + blockIdx.x * blockDim.x + threadIdx.x; r < rowEnd; r += gridDim.x * blockDim.x)
        mcRowUpdate(r, pos, sliceBase, col, val, diag, b, psi);
}

__global__ void __launch_bounds__(1024) mcSmoothSmall(int nColours, const int* __restrict__ colourStart, int nSweeps,
                                                      int symmetric, const int* __restrict__ pos,
                                                      const int* __restrict__ sliceBase, const int* __restrict__ col,
                                                      const float* __restrict__ val, const float* __restrict__ diag,
                                                      const float* __restrict__ b, float* __restrict__ psi)
{
    const int steps = symmetric ? 2 * nColours : nColours;
    for (int sw = 0; sw < nSweeps; ++sw)
        for (int i = 0; i < steps; ++i)
        {
            const int k = i < nColours ? i : 2 * nColours - 1 - i;  // symmetric: the colours back again
            const int e = colourStart[k + 1];
            for (int r = colourStart[k] + threadIdx.x; r < e; r += blockDim.x)
                mcRowUpdate(r, pos, sliceBase, col, val, diag, b, psi);
            __syncthreads();
        }
}

__global__ void __launch_bounds__(1024) mcSmoothCluster(int nColours, const int* __restrict__ colourStart,
                                                        int nSweeps, int symmetric, const int* __restrict__ pos,
                                                        const int* __restrict__ sliceBase, const int* __restrict__ col,
                                                        const float* __restrict__ val, const float* __restrict__ diag,
                                                        const float* __restrict__ b, float* __restrict__ psi)
{
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    const int steps = symmetric ? 2 * nColours : nColours;
    for (int sw = 0; sw < nSweeps; ++sw)
        for (int i = 0; i < steps; ++i)
        {
            const int k = i < nColours ? i : 2 * nColours - 1 - i;
            const int e = colourStart[k + 1];
            for (int r = colourStart[k] + t; r < e; r += stride) mcRowUpdate(r, pos, sliceBase, col, val, diag, b, psi);
            cluster.sync();  // every thread of every CTA, once per colour
        }
}

// One smoothing call of the exact Gauss-Seidel on a small one-part level in ONE block: psi of the
// whole level in shared memory, the positions walked depth by depth (the part's positions run by
// depth) with a block barrier between depths. A cell's lower-index neighbours have smaller depths (new
// values by then) and its higher-index neighbours larger ones (still old), so each row reads what the
// sequential sweep reads and computes it with the same rounding in the same order: the source minus
// the row's terms in row order, then the division. Row data do not depend on psi, so each thread
// loads its next depth's row into registers, and the row bounds one depth further ahead, before it
// computes the current one: the chain per depth is the shared-memory gathers, the row's arithmetic
// and the barrier. Cells beyond the block's width at a depth are computed straight from memory.
constexpr int kResidentK = 16;         // row entries a thread holds in registers
constexpr int kResidentMaxBlock = 256;

template <class T>
struct ResidentRow
{
    int p;  // position, -1: none at this depth
    int w;  // entries
    int e0;
    T b, d;
    T v[kResidentK];
    int c[kResidentK];
};

template <class T>
__device__ __forceinline__ void residentLoad(const Rows<T>& A, const T* __restrict__ b, int p, int e0, int e1,
                                             ResidentRow<T>& r)
{
    r.p = p;
    r.w = 0;
    if (p < 0) return;
    r.e0 = e0;
    r.w = e1 - e0;
    r.b = b[p];
    r.d = A.diag[p];
#pragma unroll
    for (int q = 0; q < kResidentK; ++q)
        if (q < r.w)
        {
            r.v[q] = A.val[e0 + q];
            r.c[q] = A.col[e0 + q];
        }
}

template <class T>
__device__ __forceinline__ void residentRow(const Rows<T>& A, const ResidentRow<T>& r, T* x)
{
    T acc = r.b;
#pragma unroll
    for (int q = 0; q < kResidentK; ++q)
        if (q < r.w) acc = subRn(acc, mulRn(r.v[q], x[r.c[q]]));
    for (int q = kResidentK; q < r.w; ++q) acc = subRn(acc, mulRn(A.val[r.e0 + q], x[A.col[r.e0 + q]]));
    x[r.p] = divRn(acc, r.d);
}

template <class T>
__global__ void __launch_bounds__(kResidentMaxBlock) gsResident(Rows<T> A, int nDepth, const int* __restrict__ depthStart,
                                                                const T* __restrict__ b, T* __restrict__ psi, int nSweeps)
{
    extern __shared__ __align__(16) unsigned char residentSm[];
    T* x = reinterpret_cast<T*>(residentSm);
    int* ds = reinterpret_cast<int*>(residentSm + sizeof(T) * static_cast<size_t>(A.n));
    const int t = threadIdx.x;
    const int B = blockDim.x;
    for (int i = t; i < A.n; i += B) x[i] = psi[i];
    for (int i = t; i <= nDepth; i += B) ds[i] = depthStart[i];
    __syncthreads();
    for (int sw = 0; sw < nSweeps; ++sw)
    {
        ResidentRow<T> cur, nxt;
        {
            const int p = nDepth > 0 && ds[0] + t < ds[1] ? ds[0] + t : -1;
            residentLoad(A, b, p, p >= 0 ? A.rowStart[p] : 0, p >= 0 ? A.rowStart[p + 1] : 0, cur);
        }
        int pn = -1, en0 = 0, en1 = 0;
        if (nDepth > 1 && ds[1] + t < ds[2])
        {
            pn = ds[1] + t;
            en0 = A.rowStart[pn];
            en1 = A.rowStart[pn + 1];
        }
        for (int d = 0; d < nDepth; ++d)
        {
            // the next depth's row (its bounds were loaded a depth ago) and the bounds after it
            residentLoad(A, b, pn, en0, en1, nxt);
            int pf = -1, ef0 = 0, ef1 = 0;
            if (d + 2 < nDepth && ds[d + 2] + t < ds[d + 3])
            {
                pf = ds[d + 2] + t;
                ef0 = A.rowStart[pf];
                ef1 = A.rowStart[pf + 1];
            }
            if (cur.p >= 0) residentRow(A, cur, x);
            for (int p = ds[d] + t + B; p < ds[d + 1]; p += B)
            {
                T acc = b[p];
                for (int e = A.rowStart[p]; e < A.rowStart[p + 1]; ++e) acc = subRn(acc, mulRn(A.val[e], x[A.col[e]]));
                x[p] = divRn(acc, A.diag[p]);
            }
            __syncthreads();
            cur = nxt;
            pn = pf;
            en0 = ef0;
            en1 = ef1;
        }
    }
    __syncthreads();
    for (int i = t; i < A.n; i += B) psi[i] = x[i];
}

// symGaussSeidel: bPrime = source minus the row's first (neighbour-of) terms, in the reversed
// positions with psi beside it
template <class T>
__global__ void symPrepare(Rows<T> A, const int* __restrict__ posCell, const int* __restrict__ losortStart,
                           const int* __restrict__ revPos, const T* __restrict__ src, const T* __restrict__ psi,
                           T* __restrict__ bRev, T* __restrict__ xRev)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < A.n; p += gridDim.x * blockDim.x)
    {
        const int c = posCell[p];
        const int e0 = A.rowStart[p];
        const int e1 = e0 + (losortStart[c + 1] - losortStart[c]);
        T acc = src[p];
        for (int e = e0; e < e1; ++e) acc = subRn(acc, mulRn(A.val[e], psi[A.col[e]]));
        const int q = revPos[p];
        bRev[q] = acc;
        xRev[q] = psi[p];
    }
}

template <class T>
__global__ void symFinish(int n, const int* __restrict__ revPos, const T* __restrict__ xRev, T* __restrict__ psi)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) psi[p] = xRev[revPos[p]];
}

// DIC: w0 = r * rD at the lower-only level's positions (source and starting psi of the forward
// substitution)
template <class T>
__global__ void dicStart(int n, const T* __restrict__ r, const T* __restrict__ rdPos, const int* __restrict__ toLo,
                         T* __restrict__ bLo, T* __restrict__ xLo)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    {
        const T w = mulRn(r[p], rdPos[p]);
        const int q = toLo[p];
        bLo[q] = w;
        xLo[q] = w;
    }
}

// DIC: the forward substitution's result moved to the descending reversed level's positions
template <class T>
__global__ void dicMid(int n, const int* __restrict__ toLo, const int* __restrict__ toUp, const T* __restrict__ xLo,
                       T* __restrict__ bUp, T* __restrict__ xUp)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    {
        const T w = xLo[toLo[p]];
        const int q = toUp[p];
        bUp[q] = w;
        xUp[q] = w;
    }
}

// DIC: psi += w
template <class T>
__global__ void dicAdd(int n, const int* __restrict__ toUp, const T* __restrict__ xUp, T* __restrict__ psi)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        psi[p] = addRn(psi[p], xUp[toUp[p]]);
}

// per face rD[cell]*coef (the substitution's coefficient for the row of `cell`: the neighbour in the
// forward substitution, the owner in the backward one)
__global__ void dicFaceVals(int nF, const int* __restrict__ lower, const int* __restrict__ upper,
                            const double* __restrict__ coef, const double* __restrict__ rD, double* __restrict__ lo,
                            double* __restrict__ up)
{
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nF; f += gridDim.x * blockDim.x)
    {
        lo[f] = __dmul_rn(rD[upper[f]], coef[f]);
        up[f] = __dmul_rn(rD[lower[f]], coef[f]);
    }
}

template <class T>
__global__ void byPosition(int n, const int* __restrict__ posCell, const double* __restrict__ byCell, T* __restrict__ out)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        out[p] = static_cast<T>(byCell[posCell[p]]);
}

template <class T>
__global__ void fillValue(long long n, T* __restrict__ x, T v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = v;
}

// the diagonal by reversed position (cell n-1-c of the reversed level is cell c)
template <class T>
__global__ void revDiag(int n, const int* __restrict__ posCellR, const double* __restrict__ diag, T* __restrict__ out)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        out[q] = static_cast<T>(diag[n - 1 - posCellR[q]]);
}

__global__ void mcValues(long long nEnt, int nRows, const int* __restrict__ face, const int* __restrict__ pos,
                         const double* __restrict__ upper, const float* __restrict__ posDiag, float* __restrict__ val,
                         float* __restrict__ diag)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nEnt; i += stride)
    {
        const int f = face[i];
        val[i] = f >= 0 ? static_cast<float>(upper[f]) : 0.0f;
        if (i < nRows)
        {
            const int p = pos[i];
            diag[i] = p >= 0 ? posDiag[p] : 1.0f;
        }
    }
}

}  // namespace k

// The sweep's shared-memory ceiling, raised once per device and value type before the first launch
// (outside any stream capture: the matrix constructor calls it).
template <class T>
void allowSweepSmem(int device)
{
    static std::atomic<unsigned long long> done[2]{};
    const unsigned long long bit = 1ull << (device & 63);
    std::atomic<unsigned long long>& d = done[sizeof(T) == 8 ? 0 : 1];
    if (d.load() & bit) return;
    B2G_CUDA(cudaFuncSetAttribute(k::gsSweep<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024));
    B2G_CUDA(cudaFuncSetAttribute(k::gsResident<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kResidentSmem)));
    constexpr int denseSmem = static_cast<int>(sizeof(double)) * k::kDenseMax * k::kDenseMax;
    B2G_CUDA(cudaFuncSetAttribute(k::coarseDenseSolve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, denseSmem));
    B2G_CUDA(cudaFuncSetAttribute(k::coarseDenseFactor, cudaFuncAttributeMaxDynamicSharedMemorySize, denseSmem));
    d.fetch_or(bit);
}

cudaEvent_t Matrix::timedBegin(int kind, int level, int units)
{
    if (!g_profiling) return nullptr;
    std::pair<cudaEvent_t, cudaEvent_t> e;
    if (!evFree.empty())
    {
        e = evFree.back();
        evFree.pop_back();
    }
    else
    {
        B2G_CUDA(cudaEventCreate(&e.first));
        B2G_CUDA(cudaEventCreate(&e.second));
    }
    TimedRegion r;
    r.start = e.first;
    r.end = e.second;
    r.kind = kind;
    r.level = level;
    r.units = units;
    if (capturing)
    {
        // an event-record node in the graph, re-recorded by every replay
        B2G_CUDA(cudaEventRecordWithFlags(r.start, stream, cudaEventRecordExternal));
        capturing->regions.push_back(r);
    }
    else
    {
        B2G_CUDA(cudaEventRecord(r.start, stream));
        evOpen.push_back(r);
    }
    return r.start;
}

// regions never nest: the one being closed is the last one opened
void Matrix::timedEnd(cudaEvent_t start)
{
    if (!start) return;
    if (capturing)
        B2G_CUDA(cudaEventRecordWithFlags(capturing->regions.back().end, stream, cudaEventRecordExternal));
    else
        B2G_CUDA(cudaEventRecord(evOpen.back().end, stream));
}

void Matrix::addRegion(const TimedRegion& r)
{
    float x = 0.f;
    B2G_CUDA(cudaEventElapsedTime(&x, r.start, r.end));
    const size_t need = static_cast<size_t>(r.level) + 1;
    for (int k = 0; k < 3; ++k)
        if (lvMs[k].size() < need)
        {
            lvMs[k].resize(need, 0.0);
            lvCalls[k].resize(need, 0);
            lvUnits[k].resize(need, 0);
        }
    lvMs[r.kind][r.level] += x;
    lvCalls[r.kind][r.level] += 1;
    lvUnits[r.kind][r.level] += r.units;
}

void Matrix::collectGraphTimings(IterationGraph& G)
{
    if (!g_profiling) return;
    for (const TimedRegion& r : G.regions) addRegion(r);
}

void Matrix::releaseGraph(IterationGraph& G)
{
    if (G.exec) cudaGraphExecDestroy(G.exec);
    G.exec = nullptr;
    for (const TimedRegion& r : G.regions) evFree.emplace_back(r.start, r.end);
    G.regions.clear();
}

void Matrix::timingsBegin()
{
    for (int i = 0; i < 4; ++i)
    {
        ms[i] = 0;
        counts[i] = 0;
    }
    launches = 0;
    for (int k = 0; k < 3; ++k)
    {
        lvMs[k].clear();
        lvCalls[k].clear();
        lvUnits[k].clear();
    }
    if (!g_profiling) return;
    if (!evSolve[0])
    {
        B2G_CUDA(cudaEventCreate(&evSolve[0]));
        B2G_CUDA(cudaEventCreate(&evSolve[1]));
    }
    B2G_CUDA(cudaEventRecord(evSolve[0], stream));
}

void Matrix::timingsEnd()
{
    counts[3] = launches;
    if (!g_profiling) return;
    B2G_CUDA(cudaEventRecord(evSolve[1], stream));
    B2G_CUDA(cudaEventSynchronize(evSolve[1]));
    float t = 0.f;
    B2G_CUDA(cudaEventElapsedTime(&t, evSolve[0], evSolve[1]));
    ms[3] = t;
    for (const TimedRegion& r : evOpen)
    {
        addRegion(r);
        evFree.emplace_back(r.start, r.end);
    }
    evOpen.clear();
    for (int k = 0; k < 2; ++k)
        if (!lvMs[k].empty())
        {
            ms[k] = lvMs[k][0];
            counts[k] = lvUnits[k][0];
        }
    ms[2] = ms[3] - ms[0] - ms[1];
    long long regions = 0;
    for (int k = 0; k < 3; ++k)
        if (!lvCalls[k].empty()) regions += lvCalls[k][0];
    counts[2] = counts[3] - regions;
}

Matrix::~Matrix()
{
    for (IterationGraph* g : {&pcgGraph, &gamgGraph}) releaseGraph(*g);
    for (const TimedRegion& r : evOpen) evFree.emplace_back(r.start, r.end);
    for (auto& e : evFree)
    {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (evSolve[0])
    {
        cudaEventDestroy(evSolve[0]);
        cudaEventDestroy(evSolve[1]);
    }
    if (sideStream)
    {
        cudaStreamSynchronize(sideStream);
        cudaEventDestroy(sideEv[0]);
        cudaEventDestroy(sideEv[1]);
        cudaStreamDestroy(sideStream);
    }
}

template <> VCycleData<double>& Matrix::data<double>() { return v64; }
template <> VCycleData<float>& Matrix::data<float>() { return v32; }

Matrix::Matrix(Mesh* m, cudaStream_t s) : mesh(m), stream(s)
{
    const size_t n0 = nAlloc(0);
    for (DBuf<double>* b : {&psi, &source, &rA, &wA, &pA, &AwA, &fc, &fr}) b->alloc(n0, s);
    scal.alloc(1, s);
    scal.zero(s);
    // reductions run before the coarse levels exist (the initial residual and normFactor)
    v64.partial.alloc(2 * kMaxPartials, s);
    v64.sf.alloc(1, s);
    err.alloc(1, s);
    err.zero(s);
    coarseCount.alloc(1, s);
    coarseCount.zero(s);
    v64.coef.resize(m->lev.size());
    int dev = 0;
    B2G_CUDA(cudaGetDevice(&dev));
    allowSweepSmem<double>(dev);
    allowSweepSmem<float>(dev);
}

void Matrix::setFine(const double* diag, const double* upper, int memspace)
{
    const LevelAddr& L = mesh->lev[0];
    LevelCoef<double>& C = v64.coef[0];
    const cudaMemcpyKind kind = memspace == B2G_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    C.diag.ensure(L.nCells, stream);
    C.upper.ensure(L.nFaces, stream);
    B2G_CUDA(cudaMemcpyAsync(C.diag.p, diag, sizeof(double) * L.nCells, kind, stream));
    if (L.nFaces) B2G_CUDA(cudaMemcpyAsync(C.upper.p, upper, sizeof(double) * L.nFaces, kind, stream));
    fillGsLayout(L, C, stream);
    coarseBuilt = false;
    v32.built = false;
    ++coefGen;
}

// GamgHierarchy::build (GAMG:565-623): Galerkin coarse matrices level by level
void Matrix::buildCoarse()
{
    if (coarseBuilt) return;
    const int nL = nLevels();
    for (int i = 0; i < nL; ++i)
    {
        const Step& S = mesh->step[i];
        const LevelAddr& Cl = mesh->lev[i + 1];
        const LevelCoef<double>& F = v64.coef[i];
        LevelCoef<double>& C = v64.coef[i + 1];
        C.diag.ensure(Cl.nCells, stream);
        C.upper.ensure(Cl.nFaces, stream);
        k::galerkinDiag<<<rowsGrid(Cl.nCells), NT, 0, stream>>>(Cl.nCells, S.cellStart.p, S.cellList.p, S.intStart.p,
                                                                S.intList.p, F.diag.p, F.upper.p, C.diag.p);
        if (Cl.nFaces)
            k::galerkinUpper<<<rowsGrid(Cl.nFaces), NT, 0, stream>>>(Cl.nFaces, S.faceBeg.p, S.faceEnd.p,
                                                                     S.faceList.p, F.upper.p, C.upper.p);
        B2G_LAUNCH_CHECK();
        fillGsLayout(Cl, C, stream);
    }
    // V-cycle work
    v64.corr.resize(nL);
    v64.src.resize(nL);
    for (int i = 0; i < nL; ++i)
    {
        v64.corr[i].ensure(nAlloc(i + 1), stream);
        v64.src[i].ensure(nAlloc(i + 1), stream);
    }
    v64.ACf.ensure(nAlloc(0), stream);
    v64.preSmoothed.ensure(nAlloc(0), stream);
    const int nc = nL > 0 ? mesh->lev[nL].nCells : mesh->lev[0].nCells;
    for (DBuf<double>* b : {&v64.cpA, &v64.cwA, &v64.crA, &v64.crD}) b->ensure(std::max(nc, 1), stream);
    v64.built = true;
    coarseBuilt = true;
}

void Matrix::ensureFp32()
{
    if (v32.built) return;
    buildCoarse();
    const int nL = nLevels();
    v32.coef.resize(nL + 1);
    for (int i = 0; i <= nL; ++i)
    {
        const LevelAddr& L = mesh->lev[i];
        LevelCoef<float>& C = v32.coef[i];
        allocGsLayout(L, C, stream);
        castInto<float, double>(L.nCells, v64.coef[i].gsDiag.p, C.gsDiag.p, stream);
        castInto<float, double>(2LL * L.nFaces, v64.coef[i].rowVal.p, C.rowVal.p, stream);
        fillEll<float>(L, C, stream);
        fillBlobs<float>(L, C, v64.coef[i].upper.p, stream);
    }
    v32.corr.resize(nL);
    v32.src.resize(nL);
    for (int i = 0; i < nL; ++i)
    {
        v32.corr[i].ensure(nAlloc(i + 1), stream);
        v32.src[i].ensure(nAlloc(i + 1), stream);
    }
    const size_t n0 = nAlloc(0);
    v32.ACf.ensure(n0, stream);
    v32.preSmoothed.ensure(n0, stream);
    v32.partial.ensure(2 * kMaxPartials, stream);
    v32.sf.ensure(1, stream);
    for (DBuf<float>* b : {&r32, &w32, &AwA32, &fc32, &fr32}) b->ensure(n0, stream);
    rOld.ensure(n0, stream);
    v32.built = true;
}

template <class T>
void Matrix::toPos(int level, const T* nat, T* pos)
{
    const LevelAddr& L = mesh->lev[level];
    if (L.nCells) k::toPositions<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(L.nCells, L.gs.posCell.p, nat, pos);
    B2G_LAUNCH_CHECK();
    ++launches;
}

template <class T>
void Matrix::fromPos(int level, const T* pos, T* nat)
{
    const LevelAddr& L = mesh->lev[level];
    if (L.nCells) k::fromPositions<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(L.nCells, L.gs.posCell.p, pos, nat);
    B2G_LAUNCH_CHECK();
    ++launches;
}

double* Matrix::ioBuf(int i)
{
    if (!io[i].p) io[i].alloc(nAlloc(0), stream);
    return io[i].p;
}

template <class T>
void Matrix::amul(int level, const T* x, T* y)
{
    const LevelAddr& L = mesh->lev[level];
    cudaEvent_t e = timedBegin(0, level, 1);
    k::amul<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(rowsOf(L, data<T>().coef[level]), x, y);
    timedEnd(e);
    B2G_LAUNCH_CHECK();
    ++launches;
}

// r = source - A*psi on the finest level, Amul's rounding (fused Amul and subtract; GAMG:1098-1106)
template <class T>
void Matrix::residualBetween(const T* source, const T* x, T* r)
{
    const LevelAddr& F = mesh->lev[0];
    cudaEvent_t e = timedBegin(2, 0, 1);
    k::amulSubtract<T><<<rowsGrid(F.nCells), NT, 0, stream>>>(rowsOf(F, data<T>().coef[0]), source, x, r);
    timedEnd(e);
    B2G_LAUNCH_CHECK();
    ++launches;
}

template <class T>
void Matrix::smooth(int level, int smoother, T* psiL, const T* src, int nSweeps, unsigned long long* trace)
{
    if (nSweeps <= 0) return;
    cudaEvent_t e = timedBegin(1, level, nSweeps);
    smoothCall<T>(level, smoother, psiL, src, nSweeps, trace);
    timedEnd(e);
}

template <class T>
void Matrix::smoothCall(int level, int smoother, T* psiL, const T* src, int nSweeps, unsigned long long* trace)
{
    if (smoother < B2G_SMOOTHER_GAUSS_SEIDEL || smoother > B2G_SMOOTHER_DIC_GAUSS_SEIDEL)
        fail(B2G_ERR_ARGUMENT, "b2g: unknown smoother");
    if (smoother == B2G_SMOOTHER_DIC || smoother == B2G_SMOOTHER_DIC_GAUSS_SEIDEL)
    {
        // DICSmoother's sweeps; DICGaussSeidel then sweeps Gauss-Seidel as often (GAMG:234-317)
        if (mesh->lev[level].nCells == 0) return;
        dicSmooth<T>(level, psiL, src, nSweeps);
        if (smoother == B2G_SMOOTHER_DIC) return;
        smoother = B2G_SMOOTHER_GAUSS_SEIDEL;
    }
    const bool symmetric = smoother == B2G_SMOOTHER_SYM_GAUSS_SEIDEL;
    if (sizeof(T) == 4 && multicolour)
    {
        mcSmooth(level, reinterpret_cast<float*>(psiL), reinterpret_cast<const float*>(src), nSweeps, symmetric);
        return;
    }
    if (mesh->lev[level].nCells == 0) return;
    const LevelAddr& L = mesh->lev[level];
    VCycleData<T>& D = data<T>();
    if (D.coef[level].pairVal.p && L.pair.nFaces > 0)
    {
        // the pair enters the Gauss-Seidel smoothers through bPrime, once per smooth() call, from psi
        // as it stands (GAMG:287-305); the sweeps then run on bPrime
        if (D.pairB.size() <= static_cast<size_t>(level)) D.pairB.resize(level + 1);
        if (!D.pairB[level].p) D.pairB[level].alloc(nAlloc(level), stream);
        k::pairFold<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(rowsOf(L, D.coef[level]), src, psiL,
                                                               D.pairB[level].p);
        B2G_LAUNCH_CHECK();
        ++launches;
        src = D.pairB[level].p;
    }
    if (symmetric)
    {
        symSmooth<T>(level, psiL, src, nSweeps);
        return;
    }
    if (!trace && pipeSweeps<T>(level, psiL, src, nSweeps)) return;
    if (!trace && level > 0 && residentSweeps<T>(level, psiL, src, nSweeps)) return;
    for (int sw = 0; sw < nSweeps; ++sw) gsLaunch<T>(mesh->lev[level], data<T>().coef[level], psiL, src, trace, level == 0);
}

// One exact Gauss-Seidel sweep of level L (its schedule) with coefficients C.
template <class T>
void Matrix::gsLaunch(const LevelAddr& L, const LevelCoef<T>& C, T* psiL, const T* src, unsigned long long* trace,
                      bool timed)
{
    const GsSchedule& G = L.gs;
    k::GsArgs<T> a;
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
    a.b = src;
    a.psi = psiL;
    a.progress = G.progress.p;
    a.ticket = reinterpret_cast<int*>(G.progress.p + static_cast<size_t>(G.nParts) * k::kProgressStride);
    a.items = 0;
    a.spinLimit = spinLimit;
    a.publish = publish;
    a.err = err.p;
    a.trace = trace;
    a.traceDepths = G.maxDepth + 2;
    const size_t smem = k::gsSmemBytes<T>(G.maxCells, G.maxEnt, G.maxGat);
    B2G_CUDA(cudaMemsetAsync(G.progress.p, 0, G.progress.bytes(), stream));
    (void)timed;
    k::gsSweep<T><<<G.nParts, G.maxCells + 128, smem, stream>>>(a);
    B2G_LAUNCH_CHECK();
    launches += 1;
}

// The reversed layout of one level in T (once per matrix): the mesh's reversed level, the diagonal
// by reversed position and the chunk blobs with this matrix's coefficients; the scratch vectors.
template <class T>
void Matrix::ensureSym(int level)
{
    VCycleData<T>& D = data<T>();
    if (static_cast<int>(D.rev.size()) <= level) D.rev.resize(mesh->lev.size());
    if (static_cast<int>(D.revB.size()) <= level)
    {
        D.revB.resize(mesh->lev.size());
        D.revX.resize(mesh->lev.size());
    }
    if (D.revGen.size() < mesh->lev.size()) D.revGen.resize(mesh->lev.size(), -1);
    if (D.rev[level].blob.p && D.revGen[level] == coefGen) return;
    LevelAddr& L = mesh->lev[level];
    buildReversedLevel(L, stream);
    const LevelAddr& R = *L.rev;
    LevelCoef<T>& C = D.rev[level];
    allocGsLayout(R, C, stream);
    k::revDiag<T><<<rowsGrid(R.nCells), NT, 0, stream>>>(R.nCells, R.gs.posCell.p, v64.coef[level].diag.p, C.gsDiag.p);
    B2G_LAUNCH_CHECK();
    fillBlobs<T>(R, C, v64.coef[level].upper.p, stream);
    D.revB[level].ensure(std::max(R.gs.nAlloc, 1), stream);
    D.revX[level].ensure(std::max(R.gs.nAlloc, 1), stream);
    D.revB[level].zero(stream);
    D.revX[level].zero(stream);
    D.revGen[level] = coefGen;
}

// What the smoother needs built before an iteration is captured (builds synchronise the stream).
// The resident sweep's depth ranges of `level` (mesh data, built once): only for a one-part level of
// at most kResidentMaxCells cells whose positions run by depth.
void Matrix::ensureResident(int level)
{
    LevelAddr& L = mesh->lev[level];
    LevelAddr::Resident& R = L.resident;
    if (R.built) return;
    R.built = true;
    R.ok = false;
    const int n = L.nCells;
    if (L.gs.nParts != 1 || n == 0 || n > kResidentMaxCells) return;
    const std::vector<int> depth = L.gs.depth.download(stream);
    const std::vector<int> posCell = L.gs.posCell.download(stream);
    std::vector<int> start(1, 0);
    int prev = 0;
    for (int p = 0; p < n; ++p)
    {
        const int dp = depth[posCell[p]];
        if (dp < prev) return;  // not by depth: keep the pipelined sweep
        while (static_cast<int>(start.size()) <= dp) start.push_back(p);
        prev = dp;
    }
    start.push_back(n);
    const int nDepth = static_cast<int>(start.size()) - 1;
    int width = 0;
    for (int d = 0; d < nDepth; ++d) width = std::max(width, start[d + 1] - start[d]);
    R.nDepth = nDepth;
    R.block = std::min(k::kResidentMaxBlock, std::max(64, (width + 31) / 32 * 32));
    R.start.upload(start.data(), start.size(), stream);
    B2G_CUDA(cudaStreamSynchronize(stream));
    R.ok = true;
}

// nSweeps exact Gauss-Seidel sweeps of a small one-part level in one resident block (gsResident);
// false if the level does not qualify (the caller then launches the pipelined sweep per sweep)
template <class T>
bool Matrix::residentSweeps(int level, T* psiL, const T* src, int nSweeps)
{
    LevelAddr& L = mesh->lev[level];
    if (!L.resident.built)
    {
        if (capturing) return false;
        ensureResident(level);
    }
    if (!L.resident.ok) return false;
    const size_t smem = sizeof(T) * static_cast<size_t>(L.nCells) + sizeof(int) * (L.resident.nDepth + 1);
    if (smem > kResidentSmem) return false;
    k::gsResident<T><<<1, L.resident.block, smem, stream>>>(rowsOf(L, data<T>().coef[level]), L.resident.nDepth,
                                                            L.resident.start.p, src, psiL, nSweeps);
    B2G_LAUNCH_CHECK();
    ++launches;
    return true;
}

void Matrix::prepareSmoother(const b2g_controls& c)
{
    const bool sym = c.smoother == B2G_SMOOTHER_SYM_GAUSS_SEIDEL;
    const bool dic = c.smoother == B2G_SMOOTHER_DIC || c.smoother == B2G_SMOOTHER_DIC_GAUSS_SEIDEL;
    // the pipelined launches of the Gauss-Seidel smoothing calls the V-cycle makes (finest sweeps on
    // level 0; pre- and post-sweeps of every smoothed coarse level), chosen before any capture
    const bool gsSweeps = c.smoother == B2G_SMOOTHER_GAUSS_SEIDEL || c.smoother == B2G_SMOOTHER_DIC_GAUSS_SEIDEL;
    const bool exact32 = c.precision == B2G_PRECISION_FP32_PRECOND && c.solver != B2G_SOLVER_GAMG;
    const bool exact64 = c.precision == B2G_PRECISION_FP64 || c.solver == B2G_SOLVER_GAMG;
    if (g_pipeline && gsSweeps && (exact32 || exact64))
    {
        auto want = [&](int level, int nSweeps) {
            if (nSweeps <= 0 || level > nLevels()) return;
            if (exact64) ensurePipe<double>(level, nSweeps);
            else ensurePipe<float>(level, nSweeps);
        };
        want(0, c.nFinestSweeps);
        for (int li = 0; li + 1 < nLevels(); ++li)
        {
            want(li + 1, std::min(c.nPostSweeps + c.postSweepsLevelMultiplier * li, c.maxPostSweeps));
            if (c.nPreSweeps) want(li + 1, std::min(c.nPreSweeps + c.preSweepsLevelMultiplier * li, c.maxPreSweeps));
        }
        if (exact64) refreshItems<double>();
        else refreshItems<float>();
    }
    // the multicolour form: each smoothing call the V-cycle makes as one pipelined launch over the
    // colours where that measured faster, chosen before any capture
    const bool mcSweeps = c.smoother != B2G_SMOOTHER_DIC && c.solver != B2G_SOLVER_GAMG &&
                          c.precision == B2G_PRECISION_FP32_PRECOND_MULTICOLOUR;
    if (g_pipeline && mcSweeps)
    {
        auto want = [&](int level, int nSweeps) {
            if (nSweeps > 0 && level <= nLevels()) ensureMcPipe(level, nSweeps, sym);
        };
        want(0, c.nFinestSweeps);
        for (int li = 0; li + 1 < nLevels(); ++li)
        {
            want(li + 1, std::min(c.nPostSweeps + c.postSweepsLevelMultiplier * li, c.maxPostSweeps));
            if (c.nPreSweeps) want(li + 1, std::min(c.nPreSweeps + c.preSweepsLevelMultiplier * li, c.maxPreSweeps));
        }
    }
    // the resident sweep's depth ranges of the small one-part levels, before any iteration is captured
    if (c.smoother != B2G_SMOOTHER_DIC)
        for (int i = 1; i < nLevels(); ++i) ensureResident(i);
    if (coupled && c.smoother != B2G_SMOOTHER_DIC)
    {
        // the Gauss-Seidel smoothers' bPrime per level, allocated before any iteration is captured
        if (v64.pairB.size() < static_cast<size_t>(nLevels())) v64.pairB.resize(nLevels());
        for (int i = 0; i < nLevels(); ++i)
            if (!v64.pairB[i].p) v64.pairB[i].alloc(nAlloc(i), stream);
    }
    if (!sym && !dic) return;
    const bool fp64 = c.precision == B2G_PRECISION_FP64 || c.solver == B2G_SOLVER_GAMG;
    for (int i = 0; i < nLevels(); ++i)
    {
        // the multicolour form sweeps symGaussSeidel by colour; DIC there runs in exact order
        if (sym && fp64) ensureSym<double>(i);
        else if (sym && c.precision == B2G_PRECISION_FP32_PRECOND) ensureSym<float>(i);
        if (dic && fp64) ensureDic<double>(i);
        else if (dic) ensureDic<float>(i);
    }
    B2G_CUDA(cudaStreamSynchronize(stream));
}

// DIC's layouts for one level in T (once per matrix): rD by the reference's recurrence
// (DICPreconditioner::calcReciprocalD, gamg_solver_cpp.cu:194-210) on the host, in face order;
// the substitutions' per-face coefficients; the lower-only and descending reversed levels (on the
// mesh, once) with blobs of diagonal 1; rD by position; scratch vectors.
template <class T>
void Matrix::ensureDic(int level)
{
    VCycleData<T>& D = data<T>();
    const size_t nl = mesh->lev.size();
    for (auto* v : {&D.dicLo, &D.dicUp})
        if (v->size() < nl) v->resize(nl);
    for (auto* v : {&D.rdPos, &D.dicR, &D.dicLoB, &D.dicLoX, &D.dicUpB, &D.dicUpX})
        if (v->size() < nl) v->resize(nl);
    if (D.dicGen.size() < nl) D.dicGen.resize(nl, -1);
    if (D.dicLo[level].blob.p && D.dicGen[level] == coefGen) return;
    LevelAddr& L = mesh->lev[level];
    const int n = L.nCells, nF = L.nFaces;
    if (rdCell.size() < nl) rdCell.resize(nl);
    if (rdGen.size() < nl) rdGen.resize(nl, -1);
    if (!rdCell[level].p || rdGen[level] != coefGen)
    {
        const std::vector<double> diag = v64.coef[level].diag.download(stream);
        const std::vector<double> coef = v64.coef[level].upper.download(stream);
        const std::vector<int> lo = L.lower.download(stream);
        const std::vector<int> up = L.upper.download(stream);
        std::vector<double> rD(diag);
        for (int f = 0; f < nF; ++f) rD[up[f]] -= coef[f] * coef[f] / rD[lo[f]];
        for (int c = 0; c < n; ++c) rD[c] = 1.0 / rD[c];
        rdCell[level].ensure(rD.size(), stream);
        B2G_CUDA(cudaMemcpyAsync(rdCell[level].p, rD.data(), sizeof(double) * rD.size(), cudaMemcpyHostToDevice,
                                 stream));
        B2G_CUDA(cudaStreamSynchronize(stream));  // rD is a host temporary
        rdGen[level] = coefGen;
    }
    buildLowerLevel(L, stream);
    buildReversedLevel(L, stream, true);
    DBuf<double> loVal, upVal;
    loVal.alloc(std::max(nF, 1), stream);
    upVal.alloc(std::max(nF, 1), stream);
    if (nF)
        k::dicFaceVals<<<std::min(ceilDiv(nF, NT), 8192), NT, 0, stream>>>(nF, L.lower.p, L.upper.p,
                                                                          v64.coef[level].upper.p, rdCell[level].p,
                                                                          loVal.p, upVal.p);
    B2G_LAUNCH_CHECK();
    for (int which = 0; which < 2; ++which)
    {
        const LevelAddr& R = which == 0 ? *L.lowerOnly : *L.revDesc;
        LevelCoef<T>& C = which == 0 ? D.dicLo[level] : D.dicUp[level];
        allocGsLayout(R, C, stream);
        k::fillValue<T><<<rowsGrid(n), NT, 0, stream>>>(n, C.gsDiag.p, T(1));
        B2G_LAUNCH_CHECK();
        fillBlobs<T>(R, C, which == 0 ? loVal.p : upVal.p, stream);
    }
    D.rdPos[level].ensure(nAlloc(level), stream);
    D.rdPos[level].zero(stream);
    k::byPosition<T><<<rowsGrid(n), NT, 0, stream>>>(n, L.gs.posCell.p, rdCell[level].p, D.rdPos[level].p);
    B2G_LAUNCH_CHECK();
    D.dicR[level].ensure(nAlloc(level), stream);
    for (auto* v : {&D.dicLoB, &D.dicLoX})
    {
        (*v)[level].ensure(std::max(L.lowerOnly->gs.nAlloc, 1), stream);
        (*v)[level].zero(stream);
    }
    for (auto* v : {&D.dicUpB, &D.dicUpX})
    {
        (*v)[level].ensure(std::max(L.revDesc->gs.nAlloc, 1), stream);
        (*v)[level].zero(stream);
    }
    B2G_CUDA(cudaStreamSynchronize(stream));  // loVal / upVal are read by the blob builds
    D.dicGen[level] = coefGen;
}

// DICSmoother::smooth (gamg_solver_cpp.cu:234-317): per sweep r = source - A psi, w = rD r, the two
// DIC substitutions (DICPreconditioner, :212-231) as forward sweeps of the lower-only and the
// descending reversed levels, psi += w
template <class T>
void Matrix::dicSmooth(int level, T* psiL, const T* src, int nSweeps)
{
    ensureDic<T>(level);
    const LevelAddr& L = mesh->lev[level];
    VCycleData<T>& D = data<T>();
    const int n = L.nCells;
    for (int sw = 0; sw < nSweeps; ++sw)
    {
        k::residual<T><<<rowsGrid(n), NT, 0, stream>>>(rowsOf(L, D.coef[level]), src, psiL, D.dicR[level].p);
        k::dicStart<T><<<rowsGrid(n), NT, 0, stream>>>(n, D.dicR[level].p, D.rdPos[level].p, L.lowerPos.p,
                                                       D.dicLoB[level].p, D.dicLoX[level].p);
        B2G_LAUNCH_CHECK();
        gsLaunch<T>(*L.lowerOnly, D.dicLo[level], D.dicLoX[level].p, D.dicLoB[level].p, nullptr, false);
        k::dicMid<T><<<rowsGrid(n), NT, 0, stream>>>(n, L.lowerPos.p, L.revDescPos.p, D.dicLoX[level].p,
                                                     D.dicUpB[level].p, D.dicUpX[level].p);
        B2G_LAUNCH_CHECK();
        gsLaunch<T>(*L.revDesc, D.dicUp[level], D.dicUpX[level].p, D.dicUpB[level].p, nullptr, false);
        k::dicAdd<T><<<rowsGrid(n), NT, 0, stream>>>(n, L.revDescPos.p, D.dicUpX[level].p, psiL);
        B2G_LAUNCH_CHECK();
        launches += 4;
    }
}

// symGaussSeidel sweeps (gaussSeidelSweeps' symmetric variant, smooth_solver_cpp.cu:87-166): the
// forward walk; then bPrime = source minus the faces the cell is the neighbour of times the new psi
// (subtracted in ascending face order, as the forward walk distributes them), moved with psi to the
// reversed positions; the backward walk as a forward sweep of the reversed level; psi moved back.
template <class T>
void Matrix::symSmooth(int level, T* psiL, const T* src, int nSweeps)
{
    ensureSym<T>(level);
    const LevelAddr& L = mesh->lev[level];
    VCycleData<T>& D = data<T>();
    const LevelCoef<T>& C = D.coef[level];
    for (int sw = 0; sw < nSweeps; ++sw)
    {
        gsLaunch<T>(L, C, psiL, src, nullptr, level == 0);
        k::symPrepare<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(rowsOf(L, C), L.gs.posCell.p, L.losortStart.p,
                                                               L.revPos.p, src, psiL, D.revB[level].p,
                                                               D.revX[level].p);
        B2G_LAUNCH_CHECK();
        gsLaunch<T>(*L.rev, D.rev[level], D.revX[level].p, D.revB[level].p, nullptr, level == 0);
        k::symFinish<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(L.nCells, L.revPos.p, D.revX[level].p, psiL);
        B2G_LAUNCH_CHECK();
        launches += 2;
    }
}

// Gauss-Seidel sweeps of the FP32 V-cycle, colour by colour (B2G_PRECISION_FP32_PRECOND_MULTICOLOUR);
// symmetric: each sweep takes the colours forward, then back
void Matrix::mcSmooth(int level, float* psiL, const float* src, int nSweeps, bool symmetric)
{
    const Colouring& C = mesh->lev[level].mc;
    // the call as one pipelined launch over the colours, where that measured faster (ensureMcPipe)
    const auto it = C.pipe.find(nSweeps * 2 + (symmetric ? 1 : 0));
    if (g_pipeline && it != C.pipe.end() && it->second.use)
    {
        pipeLaunch<float>(level, *it->second.sched, psiL, src, true);
        return;
    }
    mcLaunch(level, C.fused, C.cluster, C.block, psiL, src, nSweeps, true, symmetric);
}

namespace {

// The launch configuration of mcSmoothCluster: one cluster of `ctas` CTAs of 1024 threads (the grid).
struct ClusterLaunch
{
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg;
    ClusterLaunch(int ctas, cudaStream_t s)
    {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(ctas);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg = cudaLaunchConfig_t{};
        cfg.gridDim = dim3(static_cast<unsigned>(ctas));
        cfg.blockDim = dim3(1024);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
};

// Whether one cluster of `ctas` 1024-thread CTAs of mcSmoothCluster can be resident on this device
// (sizes above 8 are non-portable and need the kernel's opt-in on the current device, set here).
bool clusterFits(int ctas, cudaStream_t s)
{
    if (ctas > 8 &&
        cudaFuncSetAttribute(k::mcSmoothCluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    ClusterLaunch L(ctas, s);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k::mcSmoothCluster, &L.cfg) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return n >= 1;
}

}  // namespace

// nSweeps multicolour sweeps of one level in a given shape: one block for the whole level, one
// cluster of `cluster` CTAs for the whole level, or one launch per colour of `block` threads per block
void Matrix::mcLaunch(int level, bool fused, int cluster, int block, float* psiL, const float* src, int nSweeps,
                      bool timed, bool symmetric)
{
    const Colouring& C = mesh->lev[level].mc;
    const LevelCoef<float>& F = v32.coef[level];
    if (cluster > 0)
    {
                ClusterLaunch L(cluster, stream);
        B2G_CUDA(cudaLaunchKernelEx(&L.cfg, k::mcSmoothCluster, C.nColours, static_cast<const int*>(C.colourStartD.p),
                                    nSweeps, symmetric ? 1 : 0, static_cast<const int*>(C.pos.p),
                                    static_cast<const int*>(C.sliceBase.p), static_cast<const int*>(C.col.p),
                                    static_cast<const float*>(F.mcVal.p), static_cast<const float*>(F.mcDiag.p), src,
                                    psiL));
        ++launches;
        return;
    }
    if (fused)
    {
                k::mcSmoothSmall<<<1, 1024, 0, stream>>>(C.nColours, C.colourStartD.p, nSweeps, symmetric ? 1 : 0, C.pos.p,
                                                  C.sliceBase.p, C.col.p, F.mcVal.p, F.mcDiag.p, src, psiL);
        B2G_LAUNCH_CHECK();
        ++launches;
        return;
    }
    const int steps = symmetric ? 2 * C.nColours : C.nColours;
    for (int sw = 0; sw < nSweeps; ++sw)
        for (int i = 0; i < steps; ++i)
        {
            const int k = i < C.nColours ? i : 2 * C.nColours - 1 - i;
            const int b = C.colourStart[k], e = C.colourStart[k + 1];
            if (e <= b) continue;
                        k::mcSweep<<<std::min(ceilDiv(e - b, block), 16 * DeviceInfo::get().numSMs), block, 0, stream>>>(
                b, e, C.pos.p, C.sliceBase.p, C.col.p, F.mcVal.p, F.mcDiag.p, src, psiL);
            B2G_LAUNCH_CHECK();
            ++launches;
        }
}

// The autotuner of the multicolour sweep: times every candidate launch shape on the level's own
// layout (one block sweeping the whole level when it has at most kMcSmallRows rows; one cluster of 4,
// 8 or 16 CTAs sweeping it when it has at most kMcClusterMaxRows rows and the cluster fits the device;
// one launch per colour at 128, 256 or 512 threads per block) and keeps the fastest. Every shape
// computes each row with the same arithmetic on the same final values, so the choice changes the time
// only. Runs once per mesh level, on
// this matrix's FP32 values and scratch vectors, outside any capture.
void Matrix::tuneMulticolour(int level)
{
    Colouring& C = mesh->lev[level].mc;
    if (C.tuned) return;
    float* x = level == 0 ? w32.p : v32.corr[level - 1].p;
    float* b = level == 0 ? r32.p : v32.src[level - 1].p;
    zeroArray<float>(static_cast<long long>(nAlloc(level)), x, stream);
    castInto<float, double>(n(level), v64.coef[level].gsDiag.p, b, stream);
    struct Shape
    {
        bool fused;
        int cluster;
        int block;
    };
    std::vector<Shape> shapes;
    if (C.nRows <= k::kMcSmallRows) shapes.push_back({true, 0, 1024});
    if (C.nRows <= k::kMcClusterMaxRows)
        for (int ctas : {4, 8, 16})
            if (clusterFits(ctas, stream)) shapes.push_back({false, ctas, 1024});
    for (int bl : {128, 256, 512}) shapes.push_back({false, 0, bl});
    cudaEvent_t e0, e1;
    B2G_CUDA(cudaEventCreate(&e0));
    B2G_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    const long long l0 = launches;
    for (const Shape& sh : shapes)
    {
        mcLaunch(level, sh.fused, sh.cluster, sh.block, x, b, 1, false);  // warm
        B2G_CUDA(cudaEventRecord(e0, stream));
        mcLaunch(level, sh.fused, sh.cluster, sh.block, x, b, 3, false);
        B2G_CUDA(cudaEventRecord(e1, stream));
        B2G_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        B2G_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        ms /= 3.f;
        if (!C.tuned || ms < best)
        {
            best = ms;
            C.fused = sh.fused;
            C.cluster = sh.cluster;
            C.block = sh.block;
            C.tuned = true;
        }
    }
    launches = l0;
    C.msPerSweep = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// The multicolour layout of every level (on the mesh, once) and this matrix's FP32 values in it.
void Matrix::ensureMulticolour()
{
    ensureFp32();
    if (mcBuilt && mcGen == coefGen) return;
    for (int i = 0; i <= nLevels(); ++i)
    {
        LevelAddr& L = mesh->lev[i];
        buildColouring(L, stream);
        LevelCoef<float>& F = v32.coef[i];
        const Colouring& C = L.mc;
        F.mcVal.ensure(std::max<long long>(C.nEnt, 1), stream);
        F.mcDiag.ensure(std::max(C.nRows, 1), stream);
        const long long m = std::max<long long>(C.nEnt, C.nRows);
        if (m)
            k::mcValues<<<std::min(ceilDiv(m, NT), 8192), NT, 0, stream>>>(C.nEnt, C.nRows, C.face.p, C.pos.p,
                                                                           v64.coef[i].upper.p, F.gsDiag.p,
                                                                           F.mcVal.p, F.mcDiag.p);
        B2G_LAUNCH_CHECK();
        if (!C.tuned) tuneMulticolour(i);
    }
    mcBuilt = true;
    mcGen = coefGen;
}

template <class T>
void Matrix::scale(int level, T* field, T* Acf, const T* src)
{
    const LevelAddr& L = mesh->lev[level];
    VCycleData<T>& D = data<T>();
    if (serial && sizeof(T) == 8)
    {
        k::amul<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(rowsOf(L, D.coef[level]), field, Acf);
        k::serialScaleDots<<<1, 32, 0, stream>>>(L.nCells, reinterpret_cast<const double*>(field),
                                                 reinterpret_cast<const double*>(src),
                                                 reinterpret_cast<const double*>(Acf), L.gs.posOf.p,
                                                 reinterpret_cast<double*>(D.sf.p));
    }
    else
    {
        const int g = redGrid(L.nCells);
        cudaEvent_t e = timedBegin(2, level, 1);
        k::amulScaleDots<T, NT><<<g, NT, 0, stream>>>(rowsOf(L, D.coef[level]), field, src, Acf, D.partial.p);
        timedEnd(e);
        k::scaleFactor<T, NT><<<1, NT, 0, stream>>>(D.partial.p, g, D.sf.p);
    }
    k::scaleUpdate<T><<<rowsGrid(L.nCells), NT, 0, stream>>>(L.nCells, D.sf.p, field, src, Acf,
                                                             D.coef[level].gsDiag.p);
    B2G_LAUNCH_CHECK();
    launches += 3;
}

void Matrix::reduceInto(int op, int n, const double* a, const double* b, double* slot)
{
    if (serial)
    {
        const int* po = mesh->lev[0].gs.posOf.p;
        if (op == k::RED_DOT) k::serialReduce<k::RED_DOT><<<1, 32, 0, stream>>>(n, a, b, po, slot);
        else if (op == k::RED_SUMMAG) k::serialReduce<k::RED_SUMMAG><<<1, 32, 0, stream>>>(n, a, b, po, slot);
        else k::serialReduce<k::RED_SUM><<<1, 32, 0, stream>>>(n, a, b, po, slot);
        ++launches;
    }
    else
    {
        const int g = redGrid(n);
        if (op == k::RED_DOT) k::reducePartial<double, NT, k::RED_DOT><<<g, NT, 0, stream>>>(n, a, b, v64.partial.p);
        else if (op == k::RED_SUMMAG)
            k::reducePartial<double, NT, k::RED_SUMMAG><<<g, NT, 0, stream>>>(n, a, b, v64.partial.p);
        else k::reducePartial<double, NT, k::RED_SUM><<<g, NT, 0, stream>>>(n, a, b, v64.partial.p);
        k::reduceFinal<double, NT><<<1, NT, 0, stream>>>(v64.partial.p, g, slot);
        launches += 2;
    }
    B2G_LAUNCH_CHECK();
}

template <class T>
void Matrix::restrictTo(int step, const T* fine, T* coarse)
{
    const Step& S = mesh->step[step];
    k::restrictField<T><<<rowsGrid(S.nCoarse), NT, 0, stream>>>(S.nCoarse, S.rStartP.p, S.rListP.p, fine, coarse);
    B2G_LAUNCH_CHECK();
    ++launches;
}

template <class T>
void Matrix::prolongFrom(int step, const T* coarse, T* fine)
{
    const Step& S = mesh->step[step];
    k::prolongField<T><<<rowsGrid(S.nFine), NT, 0, stream>>>(S.nFine, S.prolongP.p, coarse, fine);
    B2G_LAUNCH_CHECK();
    ++launches;
}

template <>
void Matrix::coarsestSolve<double>(int level, double* x, const double* src, double tol, double relTol,
                                   k::DevPerf* out, bool logIt)
{
    const LevelAddr& L = mesh->lev[level];
    const LevelCoef<double>& C = v64.coef[level];
    k::CoarsestArgs<double> a;
    a.n = L.nCells;
    a.nF = L.nFaces;
    a.lower = L.lower.p;
    a.upper = L.upper.p;
    a.posOf = L.gs.posOf.p;
    a.rowStart = L.gs.posRow.p;
    a.col = L.gs.entColPos.p;
    a.val = C.rowVal.p;
    a.diag = C.gsDiag.p;
    a.coef = C.upper.p;
    a.source = src;
    a.psi = x;
    a.pA = v64.cpA.p;
    a.wA = v64.cwA.p;
    a.rA = v64.crA.p;
    a.rD = v64.crD.p;
    a.tolerance = tol;
    a.relTol = relTol;
    a.maxIter = 1000;
    a.log = logIt ? coarseLog.p : nullptr;
    a.logCount = coarseCount.p;
    a.logCapacity = coarseLogCapacity;
    a.out = out;
    if (C.pairVal.p && L.pair.nFaces > 0)
    {
        a.pairStart = L.pair.start.p;
        a.pairCol = L.pair.col.p;
        a.pairVal = C.pairVal.p;
    }
    k::coarsestPcgDic<double><<<1, 32, 0, stream>>>(a);
    B2G_LAUNCH_CHECK();
    ++launches;
}

// The FP32 V-cycle solves its coarsest level in FP64 (the level has 10-20 cells; its precision is
// free): the FP32 source is widened, solved by the same PCG-DIC, and narrowed back.
// The coarsest level's dense Cholesky factor for the current coefficients (one warp on the device);
// the factor is used when every pivot was large enough.
void Matrix::ensureDense()
{
    if (denseGen == coefGen) return;
    buildCoarse();
    denseUse = false;
    denseGen = coefGen;
    const int lv = nLevels();
    const LevelAddr& L = mesh->lev[lv];
    const int n = L.nCells;
    if (n == 0 || n > k::kDenseMax) return;
    denseL.ensure(static_cast<size_t>(n) * n, stream);
    denseOk.ensure(1, stream);
    k::DenseArgs a;
    a.n = n;
    a.nF = L.nFaces;
    a.lower = L.lower.p;
    a.upper = L.upper.p;
    a.posOf = L.gs.posOf.p;
    a.diag = v64.coef[lv].gsDiag.p;
    a.coef = v64.coef[lv].upper.p;
    a.L = denseL.p;
    a.ok = denseOk.p;
    k::coarseDenseFactor<<<1, 32, sizeof(double) * n * n, stream>>>(a);
    B2G_LAUNCH_CHECK();
    int ok = 0;
    B2G_CUDA(cudaMemcpyAsync(&ok, denseOk.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    denseUse = ok != 0;
}

template <>
void Matrix::coarsestSolve<float>(int level, float* x, const float* src, float tol, float relTol,
                                  k::DevPerf* out, bool logIt)
{
    const int n = mesh->lev[level].nCells;
    if (denseNow && denseUse && denseGen == coefGen)
    {
        k::coarseDenseSolve<float><<<1, 32, sizeof(double) * n * n, stream>>>(n, denseL.p, src, x);
        B2G_LAUNCH_CHECK();
        ++launches;
        return;
    }
    double* x64 = v64.corr[level - 1].p;
    double* s64 = v64.src[level - 1].p;
    castInto<double, float>(n, src, s64, stream);
    castInto<double, float>(n, x, x64, stream);
    coarsestSolve<double>(level, x64, s64, static_cast<double>(tol), static_cast<double>(relTol), out, logIt);
    castInto<float, double>(n, x64, x, stream);
}

double Matrix::normFactor(int level, const double* x, const double* src, const double* Apsi, bool readBack)
{
    const LevelAddr& L = mesh->lev[level];
    if (serial)
    {
        k::serialNormFactor<<<1, 32, 0, stream>>>(rowsOf(L, v64.coef[level]), x, src, Apsi, L.gs.posOf.p,
                                                   &scal.p->nf);
        ++launches;
    }
    else
    {
        const int g = redGrid(L.nCells);
        reduceInto(k::RED_SUM, L.nCells, x, nullptr, &scal.p->sumPsi);
        k::normFactorPartial<double, NT><<<g, NT, 0, stream>>>(rowsOf(L, v64.coef[level]), x, src, Apsi,
                                                               &scal.p->sumPsi, v64.partial.p);
        k::reduceFinal<double, NT><<<1, NT, 0, stream>>>(v64.partial.p, g, &scal.p->nf);
        kNfFinish<<<1, 1, 0, stream>>>(scal.p);
        launches += 3;
    }
    B2G_LAUNCH_CHECK();
    double nf = 0;
    if (!readBack) return nf;
    B2G_CUDA(cudaMemcpyAsync(&nf, &scal.p->nf, sizeof(double), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    return nf;
}

// GAMGSolver::Vcycle (GAMG:627-735). psi is corrected in place; Apsi is scratch.
template <class T>
void Matrix::vcycle(const b2g_controls& c, T* x, const T* src, T* Apsi, T* fcor, const T* fres)
{
    VCycleData<T>& D = data<T>();
    const int coarsest = nLevels() - 1;
    restrictTo<T>(0, fres, D.src[0].p);
    for (int li = 0; li < coarsest; ++li)
    {
        const int lv = li + 1;
        if (c.nPreSweeps)
        {
            zeroArray<T>(n(lv), D.corr[li].p, stream);
            smooth<T>(lv, c.smoother, D.corr[li].p, D.src[li].p,
                      std::min(c.nPreSweeps + c.preSweepsLevelMultiplier * li, c.maxPreSweeps));
            if (c.scaleCorrection && li < coarsest - 1) scale<T>(lv, D.corr[li].p, D.ACf.p, D.src[li].p);
            // residual with rA aliasing the source, per cell
            k::residual<T><<<rowsGrid(n(lv)), NT, 0, stream>>>(rowsOf(mesh->lev[lv], D.coef[lv]), D.src[li].p,
                                                               D.corr[li].p, D.src[li].p);
            B2G_LAUNCH_CHECK();
        }
        restrictTo<T>(li + 1, D.src[li].p, D.src[li + 1].p);
    }
    zeroArray<T>(n(coarsest + 1), D.corr[coarsest].p, stream);
    coarsestSolve<T>(coarsest + 1, D.corr[coarsest].p, D.src[coarsest].p, static_cast<T>(c.precTolerance),
                     static_cast<T>(c.precRelTol), nullptr, coarseLogCapacity > 0);
    for (int li = coarsest - 1; li >= 0; --li)
    {
        const int lv = li + 1;
        if (c.nPreSweeps)
            B2G_CUDA(cudaMemcpyAsync(D.preSmoothed.p, D.corr[li].p, sizeof(T) * n(lv), cudaMemcpyDeviceToDevice,
                                     stream));
        prolongFrom<T>(li + 1, D.corr[li + 1].p, D.corr[li].p);
        if (c.scaleCorrection && li < coarsest - 1) scale<T>(lv, D.corr[li].p, D.ACf.p, D.src[li].p);
        if (c.nPreSweeps)
        {
            k::addInPlace<T><<<rowsGrid(n(lv)), NT, 0, stream>>>(n(lv), D.corr[li].p, D.preSmoothed.p);
            B2G_LAUNCH_CHECK();
        }
        smooth<T>(lv, c.smoother, D.corr[li].p, D.src[li].p,
                  std::min(c.nPostSweeps + c.postSweepsLevelMultiplier * li, c.maxPostSweeps));
    }
    const LevelAddr& F = mesh->lev[0];
    if (c.scaleCorrection && !(serial && sizeof(T) == 8) && !(D.coef[0].pairVal.p && F.pair.nFaces > 0))
    {
        // prolong, scale and correct without storing the prolonged correction (bit for bit the same)
        const Step& S0 = mesh->step[0];
        const int g = redGrid(F.nCells);
        cudaEvent_t e = timedBegin(2, 0, 1);
        k::amulScaleDotsProlong<T, NT><<<g, NT, 0, stream>>>(rowsOf(F, D.coef[0]), S0.prolongP.p,
                                                             F.gs.ellColCoarse.p, D.corr[0].p, fres,
                                                             Apsi, D.partial.p);
        timedEnd(e);
        k::scaleFactor<T, NT><<<1, NT, 0, stream>>>(D.partial.p, g, D.sf.p);
        k::scaleUpdateAddProlong<T><<<rowsGrid(F.nCells), NT, 0, stream>>>(F.nCells, D.sf.p, S0.prolongP.p,
                                                                          D.corr[0].p, fres, Apsi,
                                                                          D.coef[0].gsDiag.p, x);
        B2G_LAUNCH_CHECK();
        launches += 3;
        smooth<T>(0, c.smoother, x, src, c.nFinestSweeps);
        return;
    }
    prolongFrom<T>(0, D.corr[0].p, fcor);
    if (c.scaleCorrection)
    {
        if (serial && sizeof(T) == 8)
        {
            k::amul<T><<<rowsGrid(F.nCells), NT, 0, stream>>>(rowsOf(F, D.coef[0]), fcor, Apsi);
            k::serialScaleDots<<<1, 32, 0, stream>>>(F.nCells, reinterpret_cast<const double*>(fcor),
                                                     reinterpret_cast<const double*>(fres),
                                                     reinterpret_cast<const double*>(Apsi), F.gs.posOf.p,
                                                     reinterpret_cast<double*>(D.sf.p));
        }
        else
        {
            const int g = redGrid(F.nCells);
            cudaEvent_t e = timedBegin(2, 0, 1);
            k::amulScaleDots<T, NT><<<g, NT, 0, stream>>>(rowsOf(F, D.coef[0]), fcor, fres, Apsi, D.partial.p);
            timedEnd(e);
            k::scaleFactor<T, NT><<<1, NT, 0, stream>>>(D.partial.p, g, D.sf.p);
        }
        k::scaleUpdateAdd<T><<<rowsGrid(F.nCells), NT, 0, stream>>>(F.nCells, D.sf.p, fcor, fres, Apsi,
                                                                   D.coef[0].gsDiag.p, x);
        launches += 3;
    }
    else
    {
        k::addInPlace<T><<<rowsGrid(F.nCells), NT, 0, stream>>>(F.nCells, x, fcor);
        ++launches;
    }
    B2G_LAUNCH_CHECK();
    smooth<T>(0, c.smoother, x, src, c.nFinestSweeps);
}

// GAMGPreconditioner::precondition (GAMG:1089-1107)
void Matrix::precondition(const b2g_controls& c, double* w, const double* r)
{
    const int n0 = n(0);
    multicolour = c.precision == B2G_PRECISION_FP32_PRECOND_MULTICOLOUR;
    if (coupled && c.precision != B2G_PRECISION_FP64)
        fail(B2G_ERR_REFUSED, "b2g: a matrix with a coupled pair is solved in the FP64 form only.");
    if (c.precision == B2G_PRECISION_FP32_PRECOND || multicolour)
    {
        if (multicolour) ensureMulticolour();
        ensureFp32();
        denseNow = c.coarsestDirect != 0;
        if (denseNow && !capturing) ensureDense();
        castInto<float, double>(n0, r, r32.p, stream);
        zeroArray<float>(n0, w32.p, stream);
        const float* frp = r32.p;
        for (int cycle = 0; cycle < c.nVcycles; ++cycle)
        {
            vcycle<float>(c, w32.p, r32.p, AwA32.p, fc32.p, frp);
            if (cycle < c.nVcycles - 1)
            {
                residualBetween<float>(r32.p, w32.p, fr32.p);
                frp = fr32.p;
            }
        }
        castInto<double, float>(n0, w32.p, w, stream);
        return;
    }
    zeroArray<double>(n0, w, stream);
    const double* frp = r;
    for (int cycle = 0; cycle < c.nVcycles; ++cycle)
    {
        vcycle<double>(c, w, r, AwA.p, fc.p, frp);
        if (cycle < c.nVcycles - 1)
        {
            residualBetween<double>(r, w, fr.p);
            frp = fr.p;
        }
    }
}

void Matrix::resetLog(int capacity)
{
    coarseLogCapacity = capacity;
    if (capacity > 0 && static_cast<int>(coarseLog.n) < capacity) coarseLog.alloc(capacity, stream);
    coarseCount.zero(stream);
}

void Matrix::readLog(b2g_solve_log* log)
{
    if (!log) return;
    int cnt = 0;
    B2G_CUDA(cudaMemcpyAsync(&cnt, coarseCount.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    log->coarsestCount = cnt;
    const int m = std::min(cnt, log->coarsestCapacity);
    if (m > 0 && log->coarsest)
    {
        std::vector<k::DevPerf> h(m);
        B2G_CUDA(cudaMemcpyAsync(h.data(), coarseLog.p, sizeof(k::DevPerf) * m, cudaMemcpyDeviceToHost, stream));
        B2G_CUDA(cudaStreamSynchronize(stream));
        for (int i = 0; i < m; ++i)
        {
            log->coarsest[i].initialResidual = h[i].initialResidual;
            log->coarsest[i].finalResidual = h[i].finalResidual;
            log->coarsest[i].nIterations = h[i].nIterations;
        }
    }
}

void Matrix::checkDeviceError()
{
    int e = 0;
    B2G_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    if (e)
    {
        err.zero(stream);
        fail(B2G_ERR_DEVICE_TIMEOUT,
             "b2g: a bounded device-side wait in the Gauss-Seidel sweep gave up; the result is invalid.");
    }
}

// The addresses of the per-level buffers an iteration's launches read and write, hashed: a graph
// captured before a buffer moved is never replayed (a rebuild with new coefficients keeps them in
// place, so the graph of the previous coefficients stays valid).
unsigned long long Matrix::layoutFingerprint() const
{
    unsigned long long h = 1469598103934665603ull;
    auto mix = [&h](const void* p) {
        h ^= reinterpret_cast<unsigned long long>(p);
        h *= 1099511628211ull;
    };
    for (const auto* b : {&psi, &source, &rA, &wA, &pA, &AwA, &fc, &fr, &rOld}) mix(b->p);
    for (const auto* b : {&r32, &w32, &AwA32, &fc32, &fr32}) mix(b->p);
    for (const auto& C : v64.coef)
        for (const void* q : {(const void*)C.gsDiag.p, (const void*)C.rowVal.p, (const void*)C.blob.p,
                              (const void*)C.ellVal.p})
            mix(q);
    for (const auto& C : v32.coef)
        for (const void* q : {(const void*)C.gsDiag.p, (const void*)C.rowVal.p, (const void*)C.blob.p,
                              (const void*)C.mcVal.p, (const void*)C.mcDiag.p, (const void*)C.ellVal.p})
            mix(q);
    for (const auto& b : v64.corr) mix(b.p);
    for (const auto& b : v64.src) mix(b.p);
    for (const auto& b : v32.corr) mix(b.p);
    for (const auto& b : v32.src) mix(b.p);
    for (const auto* b : {&v64.ACf, &v64.preSmoothed, &v64.partial, &v64.sf, &v64.cpA, &v64.cwA, &v64.crA, &v64.crD})
        mix(b->p);
    for (const auto* b : {&v32.ACf, &v32.preSmoothed, &v32.partial, &v32.sf}) mix(b->p);
    for (const auto& kv : v64.items) mix(kv.second.blob.p);
    for (const auto& kv : v32.items) mix(kv.second.blob.p);
    for (const void* q : {(const void*)denseL.p}) mix(q);
    return h;
}

template <class F>
void Matrix::runIteration(IterationGraph& G, const b2g_controls& c, F&& body)
{
    std::vector<unsigned char> key(sizeof(b2g_controls) + sizeof(void*) + 3 * sizeof(int) +
                                   sizeof(unsigned long long));
    unsigned char* k = key.data();
    std::memcpy(k, &c, sizeof(b2g_controls));
    k += sizeof(b2g_controls);
    const void* logp = coarseLog.p;
    std::memcpy(k, &logp, sizeof(void*));
    k += sizeof(void*);
    const int flags[3] = {coarseLogCapacity, serial ? 1 : 0, (g_profiling ? 1 : 0) | (g_pipeline ? 2 : 0)};
    std::memcpy(k, flags, sizeof(flags));
    k += sizeof(flags);
    const unsigned long long fp = layoutFingerprint();
    std::memcpy(k, &fp, sizeof(fp));
    if (!G.exec || G.key != key)
    {
        releaseGraph(G);
        const long long l0 = launches;
        B2G_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        capturing = &G;
        try
        {
            body();
        }
        catch (...)
        {
            capturing = nullptr;
            cudaGraph_t dropped = nullptr;
            cudaStreamEndCapture(stream, &dropped);
            if (dropped) cudaGraphDestroy(dropped);
            throw;
        }
        capturing = nullptr;
        cudaGraph_t graph = nullptr;
        B2G_CUDA(cudaStreamEndCapture(stream, &graph));
        const cudaError_t e = cudaGraphInstantiate(&G.exec, graph, 0);
        cudaGraphDestroy(graph);
        B2G_CUDA(e);
        G.launchesPerReplay = launches - l0;
        G.key = std::move(key);
    }
    else
    {
        launches += G.launchesPerReplay;
    }
    B2G_CUDA(cudaGraphLaunch(G.exec, stream));
}

// PCG::scalarSolve with the GAMG preconditioner (pcgGamgSolveImpl, GAMG:1031-1143)
b2g_perf Matrix::pcg(const b2g_controls& c, b2g_solve_log* log)
{
    const int n0 = n(0);
    serial = c.reduction == B2G_REDUCTION_SERIAL;
    timingsBegin();
    resetLog(log ? std::max(log->coarsestCapacity, 0) : 0);
    amul<double>(0, psi.p, wA.p);
    k::subtract<double><<<rowsGrid(n0), NT, 0, stream>>>(n0, source.p, wA.p, rA.p);
    B2G_LAUNCH_CHECK();
    normFactor(0, psi.p, source.p, wA.p, false);
    const int g = redGrid(n0);
    reduceInto(k::RED_SUMMAG, n0, rA.p, nullptr, &scal.p->sumMag);
    kInitResidual<<<1, 1, 0, stream>>>(scal.p);
    B2G_LAUNCH_CHECK();
    PcgScalars hs;
    B2G_CUDA(cudaMemcpyAsync(&hs, scal.p, sizeof(hs), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    b2g_perf perf;
    perf.initialResidual = hs.initRes;
    perf.finalResidual = hs.initRes;
    perf.nIterations = 0;
    if (log) log->historyCount = 0;
    if (c.minIter <= 0 && convergedH(perf.finalResidual, perf.initialResidual, c.tolerance, c.relTol))
    {
        timingsEnd();
        return perf;
    }
    // the preconditioner, built on first use (PCG.C:111-118)
    if (nLevels() == 0)
        fail(B2G_ERR_REFUSED, "b2g GAMG: no coarse levels created, either matrix too small for GAMG or "
                              "nCellsInCoarsestLevel too large (GAMGSolver.C:333).");
    buildCoarse();
    const bool flexible = c.precision != B2G_PRECISION_FP64;
    if (flexible) ensureFp32();
    if (flexible && c.coarsestDirect) ensureDense();
    if (c.precision == B2G_PRECISION_FP32_PRECOND_MULTICOLOUR) ensureMulticolour();
    prepareSmoother(c);
    kPcgStart<<<1, 1, 0, stream>>>(scal.p);
    B2G_LAUNCH_CHECK();
    do
    {
        runIteration(pcgGraph, c, [&] {
            precondition(c, wA.p, rA.p);
            reduceInto(k::RED_DOT, n0, wA.p, rA.p, &scal.p->wArA);
            if (flexible) reduceInto(k::RED_DOT, n0, wA.p, rOld.p, &scal.p->wrOld);
            kPUpdate<<<rowsGrid(n0), NT, 0, stream>>>(n0, wA.p, pA.p, scal.p, flexible ? 1 : 0);
            B2G_LAUNCH_CHECK();
            amul<double>(0, pA.p, wA.p);
            reduceInto(k::RED_DOT, n0, wA.p, pA.p, &scal.p->wApA);
            kAlphaUpdate<NT><<<g, NT, 0, stream>>>(n0, psi.p, pA.p, rA.p, wA.p, flexible ? rOld.p : nullptr,
                                                  scal.p, v64.partial.p);
            if (serial) reduceInto(k::RED_SUMMAG, n0, rA.p, nullptr, &scal.p->sumMag);
            else k::reduceFinal<double, NT><<<1, NT, 0, stream>>>(v64.partial.p, g, &scal.p->sumMag);
            kIterFinish<<<1, 1, 0, stream>>>(scal.p);
            B2G_LAUNCH_CHECK();
            launches += 9;
        });
        B2G_CUDA(cudaMemcpyAsync(&hs, scal.p, sizeof(hs), cudaMemcpyDeviceToHost, stream));
        B2G_CUDA(cudaStreamSynchronize(stream));
        collectGraphTimings(pcgGraph);
        if (hs.singular) break;
        perf.finalResidual = hs.finalRes;
        if (log && log->history && perf.nIterations < log->historyCapacity)
            log->history[perf.nIterations] = hs.finalRes;
        ++perf.nIterations;
        if (log) log->historyCount = perf.nIterations;
    } while ((perf.nIterations < c.maxIter &&
              !convergedH(perf.finalResidual, perf.initialResidual, c.tolerance, c.relTol)) ||
             perf.nIterations < c.minIter);
    timingsEnd();
    checkDeviceError();
    readLog(log);
    return perf;
}

// gamgSolveFoldedImpl (GAMG:961-1027): the standalone GAMG solver
b2g_perf Matrix::gamg(const b2g_controls& c, b2g_solve_log* log)
{
    const int n0 = n(0);
    serial = c.reduction == B2G_REDUCTION_SERIAL;
    timingsBegin();
    if (nLevels() == 0)
        fail(B2G_ERR_REFUSED, "b2g GAMG: no coarse levels created, either matrix too small for GAMG or "
                              "nCellsInCoarsestLevel too large (GAMGSolver.C:333).");
    resetLog(log ? std::max(log->coarsestCapacity, 0) : 0);
    buildCoarse();
    prepareSmoother(c);
    b2g_controls cc = c;
    // the standalone solver's coarsest level runs to the GAMG entry's own tolerance and relTol
    cc.precTolerance = c.tolerance;
    cc.precRelTol = c.relTol;
    amul<double>(0, psi.p, AwA.p);
    normFactor(0, psi.p, source.p, AwA.p, false);
    k::subtract<double><<<rowsGrid(n0), NT, 0, stream>>>(n0, source.p, AwA.p, fr.p);
    reduceInto(k::RED_SUMMAG, n0, fr.p, nullptr, &scal.p->sumMag);
    kInitResidual<<<1, 1, 0, stream>>>(scal.p);
    B2G_LAUNCH_CHECK();
    PcgScalars hs;
    B2G_CUDA(cudaMemcpyAsync(&hs, scal.p, sizeof(hs), cudaMemcpyDeviceToHost, stream));
    B2G_CUDA(cudaStreamSynchronize(stream));
    b2g_perf perf;
    perf.initialResidual = hs.initRes;
    perf.finalResidual = hs.initRes;
    perf.nIterations = 0;
    if (log) log->historyCount = 0;
    if (c.minIter <= 0 && convergedH(perf.finalResidual, perf.initialResidual, c.tolerance, c.relTol))
    {
        timingsEnd();
        return perf;
    }
    do
    {
        runIteration(gamgGraph, cc, [&] {
            vcycle<double>(cc, psi.p, source.p, AwA.p, fc.p, fr.p);
            amul<double>(0, psi.p, AwA.p);
            k::subtract<double><<<rowsGrid(n0), NT, 0, stream>>>(n0, source.p, AwA.p, fr.p);
            reduceInto(k::RED_SUMMAG, n0, fr.p, nullptr, &scal.p->sumMag);
            kResidualFinish<<<1, 1, 0, stream>>>(scal.p);
            B2G_LAUNCH_CHECK();
            launches += 2;
        });
        B2G_CUDA(cudaMemcpyAsync(&hs, scal.p, sizeof(hs), cudaMemcpyDeviceToHost, stream));
        B2G_CUDA(cudaStreamSynchronize(stream));
        collectGraphTimings(gamgGraph);
        perf.finalResidual = hs.finalRes;
        if (log && log->history && perf.nIterations < log->historyCapacity)
            log->history[perf.nIterations] = hs.finalRes;
        ++perf.nIterations;
        if (log) log->historyCount = perf.nIterations;
    } while ((perf.nIterations < c.maxIter &&
              !convergedH(perf.finalResidual, perf.initialResidual, c.tolerance, c.relTol)) ||
             perf.nIterations < c.minIter);
    timingsEnd();
    checkDeviceError();
    readLog(log);
    return perf;
}

template void Matrix::toPos<double>(int, const double*, double*);
template void Matrix::fromPos<double>(int, const double*, double*);
template void Matrix::amul<double>(int, const double*, double*);
template void Matrix::amul<float>(int, const float*, float*);
template void Matrix::smooth<double>(int, int, double*, const double*, int, unsigned long long*);
template void Matrix::smooth<float>(int, int, float*, const float*, int, unsigned long long*);
template void Matrix::scale<double>(int, double*, double*, const double*);
template void Matrix::restrictTo<double>(int, const double*, double*);
template void Matrix::prolongFrom<double>(int, const double*, double*);
template void Matrix::gsLaunch<double>(const LevelAddr&, const LevelCoef<double>&, double*, const double*,
                                        unsigned long long*, bool);
template void Matrix::gsLaunch<float>(const LevelAddr&, const LevelCoef<float>&, float*, const float*,
                                       unsigned long long*, bool);
template bool Matrix::residentSweeps<double>(int, double*, const double*, int);
template bool Matrix::residentSweeps<float>(int, float*, const float*, int);

}  // namespace b2g
