// pipe_kernels.cuh -- several exact Gauss-Seidel sweeps of one level in ONE launch, pipelined: sweep
// s+1 starts on a cell as soon as every value its row reads is final, instead of after the whole of
// sweep s. Bit for bit the sequential sweeps of smooth_solver_cpp.cu:87-166, sweep after sweep.
//
// THE COMBINED DAG. In sweep s cell c reads the sweep-s values of its lower neighbours (the owners of
// the faces it is the neighbour of) and the sweep-(s-1) values of its upper neighbours (the
// neighbours of the faces it owns), and it overwrites its own sweep-(s-1) value. So item (s, c) may
// run at step
//     T_s(c) = max( T_s(l) + 1 over lower l,  T_{s-1}(u) + 1 over upper u,  T_{s-1}(c) + 1 ),
// T_0(c) = depth(c). Every row then reads exactly the operands the sequential sweeps give it, and
// computes with the same rounding in the same order, so the result is the same bit for bit.
// IN PLACE is safe: a value is overwritten only by a later item of the same cell, which by the
// recurrence runs after every item that reads the value it replaces (the sweep-s readers of c's
// sweep-s value are c's upper neighbours, which (s+1, c) waits for; the sweep-s readers of c's
// sweep-(s-1) value are its lower neighbours, which (s, c) follows). Items of one step are
// independent. S sweeps then take about depth + (S-1) * lag steps instead of S * depth, lag being
// the largest depth step across a face (2 on a structured box).
//
// THE LAUNCH. psi of the level lives in shared memory for the whole smoothing call: on one CTA, or
// on the R CTAs of a thread-block cluster (R <= 16), each holding the cells of one contiguous cell
// range ("rank"). A row reads its values from the CTA that owns each one (distributed shared memory
// for another rank's), each thread computes its items of the step, and a barrier over the CTA (R = 1)
// or the cluster (release / acquire at cluster scope) separates the steps. Every CTA runs the same
// number of barriers and no data-dependent wait: the launch cannot stall (the CTAs of a cluster are
// resident together).
//
// THE GRID FORM (gsPipeGrid, levels too large for one cluster's shared memory): psi stays in global
// memory (L2), R CTAs -- all resident, the launch is cooperative -- own one contiguous cell range
// each, and after its items of step T a CTA publishes T + 1 (a release at GPU scope). Before step T
// a CTA waits until every NEIGHBOUR rank -- one owning a cell that shares a face with one of its
// cells -- has published T. That suffices both ways: every value a row of step T reads was written
// at an earlier step by its own rank or a neighbour (read after write), and every later overwrite of
// a value read at step T happens at a later step of a neighbour, which waits for this rank's step T
// first (write after read). Each wait has an iteration limit; when one runs out the error word is
// set, every CTA leaves, and the call reports a timeout.
//
// THE ROWS. An item is {position, value slot, first and end row entry}: the row is read in place
// from the level's position-order rows (no copy per sweep, so a level's rows stay in L2). Row data do
// not depend on psi, so they are loaded ahead into registers: in the shared-memory forms a thread
// loads its next step's row before it computes the current one; in the grid form it loads its item
// record two steps ahead and its row one step ahead, and its loops run to the widest row of its warp
// (a warp-wide maximum), each lane adding only its own row's entries.
#pragma once

#include "b2g_common.cuh"
#include "gs_kernels.cuh"
#include "ldu_kernels.cuh"

namespace b2g {
namespace k {

// row entries a thread holds in registers in the shared-memory forms: as many as fit beside two rows
// (20 FP64, 24 FP32); measured against 12 and 16, the longer rows of the coarse levels (a quarter of
// them past 16 entries) cost more in tail loads than the registers
template <class T> constexpr int kPipeK = sizeof(T) == 8 ? 20 : 24;
constexpr int kPipeGridK = 8;     // the same in the grid form (its 384 threads have fewer registers)
constexpr int kPipeBlock = 256;   // threads per CTA (shared-memory forms)
constexpr int kPipeGridBlock = 384;  // threads per CTA (the grid form: 168 registers, one CTA per SM)
constexpr int kPipeMaxRanks = 16;
// entries past those a thread holds in registers are loaded this many at a time in the shared-memory
// forms (as many as fit the registers left beside the rows held)
template <class T> constexpr int kPipeTail = sizeof(T) == 8 ? 4 : 8;

template <class T>
struct PipeArgs
{
    Rows<T> A;                          // the level's position-order rows (diag, val; col = the other
                                        // cell's position, which the grid form reads psi at)
    int nSteps;
    int maxLocal;                       // shared-memory slots per rank (0 in the grid form)
    const int* __restrict__ stepStart;  // [ranks][nSteps + 1] item ranges of each rank per step
    const int4* __restrict__ item;      // {position, value slot, first entry, end entry}
    const unsigned* __restrict__ entAddr;   // per row entry: owner rank << 24 | local slot of its value
                                            // (the shared-memory forms)
    const int* __restrict__ localPos;   // [ranks][maxLocal] position of each local slot
    const int* __restrict__ localCount; // [ranks]
    const T* __restrict__ b;            // by position
    T* psi;                             // by position
};

// The grid form's synchronisation.
struct PipeGridSync
{
    unsigned* progress;                 // [ranks][kProgressStride]: word 0 = the steps the rank has done
    const int* __restrict__ nbrStart;   // [ranks + 1] each rank's neighbour ranks in nbrList
    const int* __restrict__ nbrList;
    long long spinLimit;                // polls before a wait gives up
    int* err;                           // set to 1 when a wait gives up
    int publish;                        // 0: no rank publishes its progress (a test of the waits' limit)
};

template <class T, int K>
struct PipeRow
{
    int slot;   // -1: no item for this thread
    int w;      // the row's entries
    int wq;     // the widest row of the warp (warp-uniform)
    int e0;
    T b, d;
    T v[K];
    unsigned ea[K];  // each entry's value: owner rank << 24 | slot, or its position in the grid form
                     // (turned into an address at use, so that loading the next step's row never
                     // waits for its loads)
};

__device__ __forceinline__ unsigned pipeSmemAddr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned clusterRank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned mapaCluster(unsigned a, unsigned rank)
{
    unsigned d;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(rank));
    return d;
}
template <bool kCluster>
__device__ __forceinline__ double pipeLd(unsigned a, double)
{
    double v;
    if (kCluster) asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
    else asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
    return v;
}
template <bool kCluster>
__device__ __forceinline__ float pipeLd(unsigned a, float)
{
    float v;
    if (kCluster) asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    else asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ void pipeSt(unsigned a, double v) { asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory"); }
__device__ __forceinline__ void pipeSt(unsigned a, float v) { asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory"); }
// psi in the grid form: coherent at GPU scope (another SM wrote it; not from a stale L1 line)
__device__ __forceinline__ double gridLd(const double* p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ float gridLd(const float* p)
{
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}

template <bool kCluster>
__device__ __forceinline__ void pipeBarrier()
{
    if (kCluster)
    {
        asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
    else
    {
        __syncthreads();
    }
}

// the value address of an entry: its owner rank's slot, in the rank's shared memory (the same
// offset in every CTA of the launch)
template <class T, bool kCluster>
__device__ __forceinline__ unsigned pipeAddr(unsigned ea, unsigned xa)
{
    const unsigned local = xa + static_cast<unsigned>(sizeof(T)) * (ea & 0xffffffu);
    return kCluster ? mapaCluster(local, ea >> 24) : local;
}

// a row's loads once its item record is known (they wait for no load of their own); every lane of
// the warp calls it (the warp-wide width)
template <class T, int K, bool kGrid>
__device__ __forceinline__ void pipeLoadRow(const PipeArgs<T>& a, int4 it, bool has, PipeRow<T, K>& r)
{
    r.slot = has ? it.y : -1;
    r.w = has ? it.w - it.z : 0;
    r.e0 = it.z;
    r.wq = __reduce_max_sync(0xffffffffu, r.w);
    if (!has) return;
    r.b = a.b[it.x];
    r.d = a.A.diag[it.x];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        if (k >= r.wq) break;
        if (k < r.w)
        {
            r.v[k] = a.A.val[it.z + k];
            r.ea[k] = kGrid ? static_cast<unsigned>(a.A.col[it.z + k]) : a.entAddr[it.z + k];
        }
    }
}

// the shared-memory forms: a row into registers once its item record is known (no load waits for
// another)
template <class T>
__device__ __forceinline__ void pipeLoadRec(const PipeArgs<T>& a, int4 it, bool has, PipeRow<T, kPipeK<T>>& r)
{
    r.slot = has ? it.y : -1;
    r.w = has ? it.w - it.z : 0;
    r.e0 = it.z;
    if (!has) return;
    r.b = a.b[it.x];
    r.d = a.A.diag[it.x];
#pragma unroll
    for (int q = 0; q < kPipeK<T>; ++q)
        if (q < r.w)
        {
            r.v[q] = a.A.val[it.z + q];
            r.ea[q] = a.entAddr[it.z + q];
        }
}

// One term of a row: the exact sweeps subtract the rounded product (the reference's arithmetic); the
// multicolour smoother (kFma) folds it in one fused multiply-add, as its colour-by-colour kernels do.
template <bool kFma>
__device__ __forceinline__ double pipeTerm(double acc, double v, double x)
{
    return kFma ? __fma_rn(-v, x, acc) : subRn(acc, mulRn(v, x));
}
template <bool kFma>
__device__ __forceinline__ float pipeTerm(float acc, float v, float x)
{
    return kFma ? __fmaf_rn(-v, x, acc) : subRn(acc, mulRn(v, x));
}

// Entries [e, end) of a row, folded into acc in order, kPipeTail<T> at a time: the loads of a group are
// in flight together (one entry at a time, each would wait out its own load), the subtractions keep
// the row's order.
template <class T, bool kCluster, bool kFma>
__device__ __forceinline__ T pipeTail(const PipeArgs<T>& a, int e, int end, T acc, unsigned xa)
{
    for (; e < end; e += kPipeTail<T>)
    {
        T v[kPipeTail<T>], y[kPipeTail<T>];
        unsigned ea[kPipeTail<T>];
#pragma unroll
        for (int j = 0; j < kPipeTail<T>; ++j)
            if (e + j < end)
            {
                v[j] = a.A.val[e + j];
                ea[j] = a.entAddr[e + j];
            }
#pragma unroll
        for (int j = 0; j < kPipeTail<T>; ++j)
            if (e + j < end) y[j] = pipeLd<kCluster>(pipeAddr<T, kCluster>(ea[j], xa), T());
#pragma unroll
        for (int j = 0; j < kPipeTail<T>; ++j)
            if (e + j < end) acc = pipeTerm<kFma>(acc, v[j], y[j]);
    }
    return acc;
}

// the row in the reference's order: the source minus each entry's coefficient times its value, then
// the division by the diagonal
template <class T, bool kCluster, bool kFma>
__device__ __forceinline__ void pipeRow(const PipeArgs<T>& a, const PipeRow<T, kPipeK<T>>& r, unsigned xa)
{
    T x[kPipeK<T>];
#pragma unroll
    for (int q = 0; q < kPipeK<T>; ++q)
        if (q < r.w) x[q] = pipeLd<kCluster>(pipeAddr<T, kCluster>(r.ea[q], xa), T());
    T acc = r.b;
#pragma unroll
    for (int q = 0; q < kPipeK<T>; ++q)
        if (q < r.w) acc = pipeTerm<kFma>(acc, r.v[q], x[q]);
    acc = pipeTail<T, kCluster, kFma>(a, r.e0 + kPipeK<T>, r.e0 + r.w, acc, xa);
    pipeSt(xa + static_cast<unsigned>(sizeof(T)) * static_cast<unsigned>(r.slot), divRn(acc, r.d));
}

// A row straight from memory (the items beyond the block's width at a step)
template <class T, bool kCluster, bool kFma>
__device__ __forceinline__ void pipeRowDirect(const PipeArgs<T>& a, int4 it, unsigned xa)
{
    const T acc = pipeTail<T, kCluster, kFma>(a, it.z, it.w, a.b[it.x], xa);
    pipeSt(xa + static_cast<unsigned>(sizeof(T)) * static_cast<unsigned>(it.y), divRn(acc, a.A.diag[it.x]));
}

// the same row in the grid form: values from psi in global memory, the result stored there
template <class T>
__device__ __forceinline__ void pipeRowGrid(const PipeArgs<T>& a, const PipeRow<T, kPipeGridK>& r)
{
    T x[kPipeGridK];
#pragma unroll
    for (int k = 0; k < kPipeGridK; ++k)
    {
        if (k >= r.wq) break;
        if (k < r.w) x[k] = gridLd(a.psi + r.ea[k]);
    }
    T acc = r.b;
#pragma unroll
    for (int k = 0; k < kPipeGridK; ++k)
    {
        if (k >= r.wq) break;
        if (k < r.w) acc = subRn(acc, mulRn(r.v[k], x[k]));
    }
    for (int k = kPipeGridK; k < r.w; ++k) acc = subRn(acc, mulRn(a.A.val[r.e0 + k], gridLd(a.psi + a.A.col[r.e0 + k])));
    a.psi[r.slot] = divRn(acc, r.d);
}

// A row straight from memory (the grid form's items beyond the block's width at a step: rare)
template <class T>
__device__ __forceinline__ void pipeRowGridDirect(const PipeArgs<T>& a, int4 it)
{
    T acc = a.b[it.x];
    for (int e = it.z; e < it.w; ++e) acc = subRn(acc, mulRn(a.A.val[e], gridLd(a.psi + a.A.col[e])));
    a.psi[it.y] = divRn(acc, a.A.diag[it.x]);
}

// Where a rank's step table starts in the dynamic shared memory of the shared-memory forms: after its
// maxLocal values, 16-byte aligned.
__host__ __device__ constexpr size_t pipeStepTableAt(int maxLocal, size_t valueBytes)
{
    return (valueBytes * static_cast<size_t>(maxLocal) + 15) / 16 * 16;
}

// One smoothing call (all its sweeps) of one level. Grid = one cluster of R CTAs (kCluster) or one
// CTA; dynamic shared memory = maxLocal values of T, then the rank's step table. Each thread holds two
// rows (the current step's and the next's) and the item record of the step after them, so no load of
// a step waits for another load of the same step. (Unrolling the step loop by two, to swap the rows
// without a copy, needs more registers than a thread has: it spilled and was slower.)
template <class T, bool kCluster, bool kFma = false>
__device__ __forceinline__ void gsPipeBody(const PipeArgs<T>& a)
{
    extern __shared__ __align__(16) unsigned char pipeSm[];
    T* x = reinterpret_cast<T*>(pipeSm);
    int* ss = reinterpret_cast<int*>(pipeSm + pipeStepTableAt(a.maxLocal, sizeof(T)));
    const int rank = kCluster ? static_cast<int>(clusterRank()) : 0;
    const int t = threadIdx.x;
    const int B = blockDim.x;
    const unsigned xa = pipeSmemAddr(x);
    const int cnt = a.localCount[rank];
    const int* lp = a.localPos + static_cast<size_t>(rank) * a.maxLocal;
    const int* gss = a.stepStart + static_cast<size_t>(rank) * (a.nSteps + 1);
    for (int i = t; i <= a.nSteps; i += B) ss[i] = gss[i];
    for (int i = t; i < cnt; i += B) x[i] = a.psi[lp[i]];
    // every rank's psi is in place before any row reads it
    pipeBarrier<kCluster>();
    auto itemAt = [&](int T_) { return T_ < a.nSteps && ss[T_] + t < ss[T_ + 1] ? ss[T_] + t : -1; };
    const int4 none = make_int4(0, -1, 0, 0);
    PipeRow<T, kPipeK<T>> r0, r1;
    int k1 = itemAt(0);
    pipeLoadRec(a, k1 >= 0 ? a.item[k1] : none, k1 >= 0, r0);
    k1 = itemAt(1);
    int4 it1 = k1 >= 0 ? a.item[k1] : none;
    auto step = [&](int T_, const PipeRow<T, kPipeK<T>>& cur, PipeRow<T, kPipeK<T>>& nxt) {
        // the next step's row (its item record was loaded a step ago) and the record after it
        pipeLoadRec(a, it1, k1 >= 0, nxt);
        k1 = itemAt(T_ + 2);
        if (k1 >= 0) it1 = a.item[k1];
        if (cur.slot >= 0) pipeRow<T, kCluster, kFma>(a, cur, xa);
        // items beyond the block's width at this step, straight from memory
        for (int k = ss[T_] + t + B; k < ss[T_ + 1]; k += B) pipeRowDirect<T, kCluster, kFma>(a, a.item[k], xa);
        pipeBarrier<kCluster>();
    };
    for (int T_ = 0; T_ < a.nSteps; ++T_)
    {
        step(T_, r0, r1);
        r0 = r1;
    }
    // the last barrier above ordered every read of this CTA's values before the write-back; no rank
    // reads another's shared memory after it, so the CTAs may leave in any order
    for (int i = t; i < cnt; i += B) a.psi[lp[i]] = x[i];
}

// kFma: the multicolour smoother's arithmetic (its steps are the colours of a colouring schedule)
template <class T, bool kCluster, bool kFma = false>
__global__ void __launch_bounds__(kPipeBlock, 1) gsPipe(PipeArgs<T> a)
{
    gsPipeBody<T, kCluster, kFma>(a);
}

// One smoothing call of many independent cases' levels in ONE launch, each on one CTA: block i runs
// the pipelined sweeps of table[i], skipped when its case's `active` flag (may be null) is 0.
template <class T>
__global__ void __launch_bounds__(kPipeBlock, 1) gsPipeBatch(const PipeArgs<T>* __restrict__ table,
                                                             const int* __restrict__ caseOf,
                                                             const int* __restrict__ active)
{
    if (active && active[caseOf[blockIdx.x]] == 0) return;
    const PipeArgs<T> a = table[blockIdx.x];
    gsPipeBody<T, false>(a);
}

// One smoothing call of one level in the grid form: block r is rank r (all resident: a cooperative
// launch); dynamic shared memory = the rank's step table. The caller zeroes the progress words.
template <class T>
__global__ void __launch_bounds__(kPipeGridBlock, 1) gsPipeGrid(PipeArgs<T> a, PipeGridSync g)
{
    extern __shared__ __align__(16) int gridSs[];
    __shared__ int stop;
    const int rank = blockIdx.x;
    const int t = threadIdx.x;
    const int B = blockDim.x;
    const int* gss = a.stepStart + static_cast<size_t>(rank) * (a.nSteps + 1);
    for (int i = t; i <= a.nSteps; i += B) gridSs[i] = gss[i];
    if (t == 0) stop = 0;
    __syncthreads();
    const int n0 = g.nbrStart[rank], n1 = g.nbrStart[rank + 1];
    unsigned* mine = g.progress + static_cast<size_t>(rank) * kProgressStride;
    auto itemAt = [&](int T_) { return T_ < a.nSteps && gridSs[T_] + t < gridSs[T_ + 1] ? gridSs[T_] + t : -1; };
    const int4 none = make_int4(0, -1, 0, 0);
    PipeRow<T, kPipeGridK> r0, r1;
    int k1 = itemAt(0);
    pipeLoadRow<T, kPipeGridK, true>(a, k1 >= 0 ? a.item[k1] : none, k1 >= 0, r0);
    k1 = itemAt(1);
    int4 it1 = k1 >= 0 ? a.item[k1] : none;
    // one step; false when a wait gave up (every thread of the CTA sees the same)
    auto step = [&](int T_, const PipeRow<T, kPipeGridK>& cur, PipeRow<T, kPipeGridK>& nxt) -> bool {
        pipeLoadRow<T, kPipeGridK, true>(a, it1, k1 >= 0, nxt);
        k1 = itemAt(T_ + 2);
        if (k1 >= 0) it1 = a.item[k1];
        if (T_ > 0)
        {
            // every neighbour rank has done step T_ - 1
            for (int i = n0 + t; i < n1; i += B)
            {
                const unsigned* w = g.progress + static_cast<size_t>(g.nbrList[i]) * kProgressStride;
                long long spins = 0;
                while (ldAcquire(w) < static_cast<unsigned>(T_))
                {
                    if (++spins > g.spinLimit || *reinterpret_cast<volatile int*>(g.err) != 0)
                    {
                        atomicExch(g.err, 1);
                        stop = 1;
                        break;
                    }
                }
            }
            __syncthreads();
            if (stop) return false;
        }
        if (cur.slot >= 0) pipeRowGrid<T>(a, cur);
        for (int k = gridSs[T_] + t + B; k < gridSs[T_ + 1]; k += B) pipeRowGridDirect<T>(a, a.item[k]);
        // the barrier orders the CTA's psi stores before the release (release is cumulative). The last
        // thread releases: it polls no neighbour, so the release's wait for the stores to land does not
        // hold up this CTA's next polls.
        __syncthreads();
        if (t == B - 1 && g.publish) stRelease(mine, static_cast<unsigned>(T_ + 1));
        return true;
    };
    int T_ = 0;
    for (; T_ + 1 < a.nSteps; T_ += 2)
    {
        if (!step(T_, r0, r1)) return;
        if (!step(T_ + 1, r1, r0)) return;
    }
    if (T_ < a.nSteps) step(T_, r0, r1);
}

}  // namespace k
}  // namespace b2g
