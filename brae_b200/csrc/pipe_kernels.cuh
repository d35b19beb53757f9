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
// or the cluster (release / acquire at cluster scope) separates the steps. Row data do not depend on
// psi: each thread loads its next step's row into registers, and the item after it, before it
// computes the current one, so the chain per step is the shared-memory reads, the arithmetic and the
// barrier. Every CTA runs the same number of barriers and no data-dependent wait: the launch cannot
// stall (the CTAs of a cluster are resident together).
#pragma once

#include "b2g_common.cuh"
#include "ldu_kernels.cuh"

namespace b2g {
namespace k {

constexpr int kPipeK = 16;        // row entries a thread holds in registers
constexpr int kPipeBlock = 256;   // threads per CTA
constexpr int kPipeMaxRanks = 16;

template <class T>
struct PipeArgs
{
    Rows<T> A;                          // the level's position-order rows (diag, rowStart, val)
    int nSteps;
    int maxLocal;                       // shared-memory slots per rank
    const int* __restrict__ stepStart;  // [ranks][nSteps + 1] item ranges of each rank per step
    const int4* __restrict__ item;      // {position, local slot, first entry, end entry}
    const unsigned* __restrict__ entAddr;   // per row entry: owner rank << 24 | local slot of its value
    const int* __restrict__ localPos;   // [ranks][maxLocal] position of each local slot
    const int* __restrict__ localCount; // [ranks]
    const T* __restrict__ b;            // by position
    T* psi;                             // by position
};

template <class T>
struct PipeRow
{
    int slot;   // -1: no item for this thread at this step
    int w;      // entries
    int e0;
    T b, d;
    T v[kPipeK];
    unsigned ea[kPipeK];  // each entry's value: owner rank << 24 | slot (turned into an address at use,
                          // so that loading the next step's row never waits for its loads)
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

// a row's loads once its item is known (they wait for no load of their own)
template <class T>
__device__ __forceinline__ void pipeLoadRow(const PipeArgs<T>& a, const int4& it, bool has, PipeRow<T>& r)
{
    r.slot = -1;
    r.w = 0;
    if (!has) return;
    r.slot = it.y;
    r.e0 = it.z;
    r.w = it.w - it.z;
    r.b = a.b[it.x];
    r.d = a.A.diag[it.x];
#pragma unroll
    for (int q = 0; q < kPipeK; ++q)
        if (q < r.w)
        {
            r.v[q] = a.A.val[it.z + q];
            r.ea[q] = a.entAddr[it.z + q];
        }
}

template <class T>
__device__ __forceinline__ void pipeLoad(const PipeArgs<T>& a, int k, PipeRow<T>& r)
{
    const int4 it = k >= 0 ? a.item[k] : make_int4(0, -1, 0, 0);
    pipeLoadRow(a, it, k >= 0, r);
}

// the row in the reference's order: the source minus each entry's coefficient times its value, then
// the division by the diagonal
template <class T, bool kCluster>
__device__ __forceinline__ void pipeRow(const PipeArgs<T>& a, const PipeRow<T>& r, unsigned xa)
{
    T x[kPipeK];
#pragma unroll
    for (int q = 0; q < kPipeK; ++q)
        if (q < r.w) x[q] = pipeLd<kCluster>(pipeAddr<T, kCluster>(r.ea[q], xa), T());
    T acc = r.b;
#pragma unroll
    for (int q = 0; q < kPipeK; ++q)
        if (q < r.w) acc = subRn(acc, mulRn(r.v[q], x[q]));
    for (int q = kPipeK; q < r.w; ++q)
        acc = subRn(acc, mulRn(a.A.val[r.e0 + q], pipeLd<kCluster>(pipeAddr<T, kCluster>(a.entAddr[r.e0 + q], xa), T())));
    pipeSt(xa + static_cast<unsigned>(sizeof(T)) * static_cast<unsigned>(r.slot), divRn(acc, r.d));
}

// One smoothing call (all its sweeps) of one level. Grid = one cluster of R CTAs (kCluster) or one
// CTA; dynamic shared memory = maxLocal values of T.
template <class T, bool kCluster>
__device__ __forceinline__ void gsPipeBody(const PipeArgs<T>& a)
{
    extern __shared__ __align__(16) unsigned char pipeSm[];
    T* x = reinterpret_cast<T*>(pipeSm);
    const int rank = kCluster ? static_cast<int>(clusterRank()) : 0;
    const int t = threadIdx.x;
    const int B = blockDim.x;
    const unsigned xa = pipeSmemAddr(x);
    const int cnt = a.localCount[rank];
    const int* lp = a.localPos + static_cast<size_t>(rank) * a.maxLocal;
    for (int i = t; i < cnt; i += B) x[i] = a.psi[lp[i]];
    // every rank's psi is in place before any row reads it
    pipeBarrier<kCluster>();
    const int* ss = a.stepStart + static_cast<size_t>(rank) * (a.nSteps + 1);
    // a thread's item at step T is ss[T] + t when that is below ss[T + 1]. Its item record is loaded
    // two steps ahead and its row one step ahead, so that no step waits on a load chain: at step T
    // the row of step T+1 is loaded from a record that arrived a step ago, while the record of step
    // T+2 is on its way.
    auto itemAt = [&](int T_) { return T_ < a.nSteps && ss[T_] + t < ss[T_ + 1] ? ss[T_] + t : -1; };
    PipeRow<T> cur, nxt;
    pipeLoad(a, a.nSteps > 0 ? itemAt(0) : -1, cur);
    int kn = itemAt(1);
    int4 itn = kn >= 0 ? a.item[kn] : make_int4(0, -1, 0, 0);
    for (int T_ = 0; T_ < a.nSteps; ++T_)
    {
        pipeLoadRow(a, itn, kn >= 0, nxt);
        kn = itemAt(T_ + 2);
        if (kn >= 0) itn = a.item[kn];
        if (cur.slot >= 0) pipeRow<T, kCluster>(a, cur, xa);
        // items beyond the block's width at this step, straight from memory
        for (int k = ss[T_] + t + B; k < ss[T_ + 1]; k += B)
        {
            PipeRow<T> r;
            pipeLoad(a, k, r);
            pipeRow<T, kCluster>(a, r, xa);
        }
        pipeBarrier<kCluster>();
        cur = nxt;
    }
    // the last barrier above ordered every read of this CTA's values before the write-back; no rank
    // reads another's shared memory after it, so the CTAs may leave in any order
    for (int i = t; i < cnt; i += B) a.psi[lp[i]] = x[i];
}

template <class T, bool kCluster>
__global__ void __launch_bounds__(kPipeBlock, 1) gsPipe(PipeArgs<T> a)
{
    gsPipeBody<T, kCluster>(a);
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

}  // namespace k
}  // namespace b2g
