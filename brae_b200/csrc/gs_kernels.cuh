// gs_kernels.cuh -- exact Gauss-Seidel (GaussSeidelSmoother::smooth as gaussSeidelSweeps runs it,
// src/OpenFOAM/matrices/smooth_solver_cpp.cu:87-166) on the device, bit for bit.
//
// THE SWEEP IN GATHER FORM. The reference walks cells ascending; cell c's new value is
//     (((b_c - l_f1*psi'[o1]) - l_f2*psi'[o2]) ... - u_g1*psi[n1] - u_g2*psi[n2] ...) / d_c
// where f1, f2, ... are the faces c is the neighbour of, in face order (their owners o < c were
// updated earlier in the sweep and distributed into bPrime in exactly that order), and g1, g2, ...
// the faces c owns (neighbours n > c, still at their old values). Written as a gather per cell, a
// cell only needs its owners' new values: the sweep is a DAG whose depth is the cell's "level".
//
// THE SCHEDULE (part-pipelined). Cells are split into P contiguous index ranges ("parts"), one
// persistent CTA per part. A CTA walks its cells depth by depth with a block barrier between
// depths (cheap, on-SM). Before a depth it waits, with a bounded spin, for (a) every upstream part
// (holding owners of its cells) to have finished that sweep through the deepest owner it needs, and
// (b) from the second sweep on, every downstream part (holding neighbours) to have finished the
// previous sweep through the deepest neighbour it reads. Each part publishes a monotonic progress
// word "sweep s complete through depth d" with release semantics after each depth. Waits only ever
// point to a lower part in the same sweep or to any part in an earlier sweep, so they cannot form a
// cycle; several sweeps pipeline in one launch, and psi is updated in place (every reader of a
// cell's old value precedes the writer in the DAG).
//
// Bounded waits: a spin that exceeds its budget sets the error word and every later wait returns at
// once, so a broken schedule ends the kernel with an error instead of hanging the GPU.
#pragma once

#include "b2g_common.cuh"

namespace b2g {
namespace k {

template <class T>
struct GsArgs
{
    int nParts;
    int maxDepth;
    const int* __restrict__ order;
    const int* __restrict__ partLvlStart;
    const int* __restrict__ lvlStart;
    const int* __restrict__ lvlDepth;
    const int* __restrict__ lvlNeedUp;
    const int* __restrict__ lvlNeedDown;
    const int* __restrict__ depStart;
    const int* __restrict__ depList;
    const int* __restrict__ rowStart;
    const int* __restrict__ losortStart;
    const int* __restrict__ col;
    const T* __restrict__ val;
    const T* __restrict__ diag;
    const T* __restrict__ b;
    T* psi;
    unsigned* progress;
    int* err;
};

constexpr long long kSpinLimit = 1LL << 24;  // polls (~0.5-2 s with backoff) before giving up

// Waits until progress[q] >= target for q in deps[beg, end). Threads share the list. Returns after a
// block barrier.
__device__ __forceinline__ void waitParts(const int* __restrict__ depList, int beg, int end, const unsigned* progress,
                                          unsigned target, int* err)
{
    for (int i = beg + threadIdx.x; i < end; i += blockDim.x)
    {
        const int q = depList[i];
        long long it = 0;
        while (ldAcquire(&progress[q]) < target)
        {
            if (*reinterpret_cast<volatile int*>(err)) break;
            if (++it > kSpinLimit)
            {
                atomicExch(err, 1);
                break;
            }
            __nanosleep(64);
        }
    }
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(1024) gsPipelined(GsArgs<T> a, int nSweeps)
{
    const int p = blockIdx.x;
    const int P = a.nParts;
    const int lvBeg = a.partLvlStart[p];
    const int lvEnd = a.partLvlStart[p + 1];
    const int upBeg = a.depStart[p], upEnd = a.depStart[p + 1];
    const int dnBeg = a.depStart[P + p], dnEnd = a.depStart[P + p + 1];
    const unsigned stride = static_cast<unsigned>(a.maxDepth) + 2u;
    for (int s = 0; s < nSweeps; ++s)
    {
        const unsigned base = static_cast<unsigned>(s) * stride;
        if (threadIdx.x == 0)
        {
            // nothing of this part lies above its first depth
            const int first = lvBeg < lvEnd ? a.lvlDepth[lvBeg] : a.maxDepth + 1;
            if (first > 0) stRelease(&a.progress[p], base + static_cast<unsigned>(first));
        }
        for (int j = lvBeg; j < lvEnd; ++j)
        {
            const int needUp = a.lvlNeedUp[j];
            if (needUp >= 0)
                waitParts(a.depList, upBeg, upEnd, a.progress, base + static_cast<unsigned>(needUp) + 1u, a.err);
            const int needDown = a.lvlNeedDown[j];
            if (s > 0 && needDown >= 0)
                waitParts(a.depList, dnBeg, dnEnd, a.progress, base - stride + static_cast<unsigned>(needDown) + 1u,
                          a.err);
            const int i1 = a.lvlStart[j + 1];
            for (int i = a.lvlStart[j] + threadIdx.x; i < i1; i += blockDim.x)
            {
                const int c = a.order[i];
                const int rb = a.rowStart[c];
                const int re = a.rowStart[c + 1];
                T acc = a.b[c];
                for (int e = rb; e < re; ++e) acc = subRn(acc, mulRn(a.val[e], ldcg(&a.psi[a.col[e]])));
                a.psi[c] = divRn(acc, a.diag[c]);
            }
            __syncthreads();
            if (threadIdx.x == 0)
            {
                __threadfence();
                const int next = (j + 1 < lvEnd) ? a.lvlDepth[j + 1] : a.maxDepth + 1;
                stRelease(&a.progress[p], base + static_cast<unsigned>(next));
            }
        }
        if (threadIdx.x == 0 && lvBeg == lvEnd) stRelease(&a.progress[p], base + static_cast<unsigned>(a.maxDepth) + 1u);
    }
}

}  // namespace k
}  // namespace b2g
