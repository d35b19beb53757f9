// assemble.cu -- the pressure equation ahead of the solve, on the device: simpleFoam's pEqn.H stages
// 4-5 as the reference's cpu::assemblePEqn computes them (src/applications/solvers/simpleFoam/
// pEqn_cpp.cu:209-260), on an orthogonal mesh with uncoupled patches, bit for bit:
//   rAUf   = fvc::interpolate(rAU): w*rAU[own] + (1-w)*rAU[nei] per internal face, the cell's value on a
//            boundary face (fvc.cu:626-650);
//   matrix = fvm::laplacian(rAUf, p): upper = lower = deltaCoeffs*rAUf*|Sf|, diag = minus their sum in
//            face order (fvm.cuh:130-150); per boundary face internalCoeffs = rAUf*|Sf|*gIC and
//            boundaryCoeffs = -rAUf*|Sf|*gBC (fvm.cuh:40-95) with fixedValue's gIC = -deltaCoeffs and
//            gBC = value*deltaCoeffs, zeroGradient's zeros (fv_patch_field.cuh:590-602);
//   source = div(phiHbyA)*V: the flux summed per cell in face order, the boundary faces patch by patch
//            (empty patches left out), divided by V and multiplied back (fvc.cu:706-730);
//   setReference: source[ref] += diag[ref]*value, diag[ref] += diag[ref] (pEqn_cpp.cu:248-255).
// Each cell's terms are gathered in the order the reference scatters them (its faces ascending -- the
// mesh's rows -- then its boundary faces in patch order), so every sum rounds as the reference's does.
// b2g_fold_boundary then folds the patches into diag and source for the solve (foldBoundary).

#include "capi_internal.cuh"

#include <algorithm>

namespace {

__global__ void kAsmFaces(int nF, const int* __restrict__ lower, const int* __restrict__ upper,
                          const double* __restrict__ w, const double* __restrict__ dc, const double* __restrict__ magSf,
                          const double* __restrict__ rAU, double* __restrict__ coef)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const double wf = w[f];
    const double rf = __dadd_rn(__dmul_rn(wf, rAU[lower[f]]), __dmul_rn(__dsub_rn(1.0, wf), rAU[upper[f]]));
    coef[f] = __dmul_rn(__dmul_rn(dc[f], rf), magSf[f]);
}

__global__ void kAsmBoundary(int nB, const int* __restrict__ cell, const double* __restrict__ rAU,
                             const double* __restrict__ magSf, const double* __restrict__ dc,
                             const int* __restrict__ type, const double* __restrict__ value, double* __restrict__ ic,
                             double* __restrict__ bc)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    const double pGamma = __dmul_rn(rAU[cell[b]], magSf[b]);
    const bool fixed = type[b] == 1;
    const double gIC = fixed ? -dc[b] : 0.0;
    const double gBC = fixed ? __dmul_rn(value[b], dc[b]) : 0.0;
    ic[b] = __dmul_rn(pGamma, gIC);
    bc[b] = __dmul_rn(-pGamma, gBC);
}

// per cell: diag = 0 - coef of its faces in face order; the divergence in the reference's order; source
__global__ void kAsmCells(int nC, const int* __restrict__ rowStart, const int* __restrict__ entFace,
                          const int* __restrict__ lower, const double* __restrict__ coef, const double* __restrict__ phi,
                          const int* __restrict__ bStart, const int* __restrict__ bOrder, const int* __restrict__ bType,
                          const double* __restrict__ bPhi, const double* __restrict__ V, double* __restrict__ diag,
                          double* __restrict__ source)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double d = 0.0, div = 0.0;
    for (int e = rowStart[c]; e < rowStart[c + 1]; ++e)
    {
        const int f = entFace[e];
        d = __dsub_rn(d, coef[f]);
        div = lower[f] == c ? __dadd_rn(div, phi[f]) : __dsub_rn(div, phi[f]);
    }
    for (int e = bStart[c]; e < bStart[c + 1]; ++e)
    {
        const int b = bOrder[e];
        if (bType[b] != 2) div = __dadd_rn(div, bPhi[b]);
    }
    div = __ddiv_rn(div, V[c]);
    diag[c] = d;
    source[c] = __dadd_rn(0.0, __dmul_rn(div, V[c]));
}

__global__ void kAsmReference(int ref, double value, double* diag, double* source)
{
    source[ref] = __dadd_rn(source[ref], __dmul_rn(diag[ref], value));
    diag[ref] = __dadd_rn(diag[ref], diag[ref]);
}

__global__ void kAsmIota(int n, int* v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void kAsmCheck(int nB, int nC, const int* __restrict__ cell, const int* __restrict__ type, int* err)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    if (cell[b] < 0 || cell[b] >= nC) atomicOr(err, 1);
    if (type[b] < 0 || type[b] > 2) atomicOr(err, 2);
}

template <class T>
void stageIn(b2g::DBuf<T>& d, const T* src, size_t n, int memspace, cudaStream_t s)
{
    d.alloc(std::max<size_t>(n, 1), s);
    if (!n) return;
    B2G_CUDA(cudaMemcpyAsync(d.p, src, n * sizeof(T),
                             memspace == B2G_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
}

inline int blocks(long long n) { return std::max(1, b2g::ceilDiv(n, 256)); }

}  // namespace

extern "C" B2G_API b2g_status b2g_assemble_pressure(b2g_mesh* mesh, const double* weights, const double* deltaCoeffs,
                                                    const double* magSf, const double* V, const double* rAU,
                                                    const double* phiHbyA, int nBFaces, const int32_t* bFaceCells,
                                                    const double* bMagSf, const double* bDeltaCoeffs,
                                                    const int32_t* bType, const double* bValue,
                                                    const double* bPhiHbyA, int pRefCell, double pRefValue,
                                                    double* diag, double* upper, double* source,
                                                    double* internalCoeffs, double* boundaryCoeffs, int memspace,
                                                    void* stream)
{
    using b2g::capi::need;
    return b2g::capi::guarded([&] {
        need(mesh != nullptr, "b2g_assemble_pressure: null mesh");
        need(weights && deltaCoeffs && magSf && V && rAU && phiHbyA && diag && upper && source,
             "b2g_assemble_pressure: null argument");
        need(nBFaces >= 0, "b2g_assemble_pressure: nBFaces must be non-negative");
        need(nBFaces == 0 || (bFaceCells && bMagSf && bDeltaCoeffs && bType && bValue && bPhiHbyA && internalCoeffs &&
                              boundaryCoeffs),
             "b2g_assemble_pressure: null boundary array");
        need(memspace == B2G_MEM_HOST || memspace == B2G_MEM_DEVICE, "b2g_assemble_pressure: bad memspace");
        (void)stream;
        const b2g::LevelAddr& L = mesh->m.lev[0];
        const int nC = L.nCells, nF = L.nFaces;
        need(pRefCell < nC, "b2g_assemble_pressure: pRefCell beyond the mesh");
        cudaStream_t s = mesh->m.stream;
        b2g::DBuf<double> w, dc, ms, vol, rau, phi, bms, bdc, bval, bphi;
        b2g::DBuf<int> bcell, btype;
        stageIn(w, weights, nF, memspace, s);
        stageIn(dc, deltaCoeffs, nF, memspace, s);
        stageIn(ms, magSf, nF, memspace, s);
        stageIn(vol, V, nC, memspace, s);
        stageIn(rau, rAU, nC, memspace, s);
        stageIn(phi, phiHbyA, nF, memspace, s);
        stageIn(bcell, bFaceCells, nBFaces, memspace, s);
        stageIn(bms, bMagSf, nBFaces, memspace, s);
        stageIn(bdc, bDeltaCoeffs, nBFaces, memspace, s);
        stageIn(btype, bType, nBFaces, memspace, s);
        stageIn(bval, bValue, nBFaces, memspace, s);
        stageIn(bphi, bPhiHbyA, nBFaces, memspace, s);
        b2g::DBuf<int> err;
        err.alloc(1, s);
        err.zero(s);
        if (nBFaces) kAsmCheck<<<blocks(nBFaces), 256, 0, s>>>(nBFaces, nC, bcell.p, btype.p, err.p);
        B2G_LAUNCH_CHECK();
        int e = 0;
        B2G_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        B2G_CUDA(cudaStreamSynchronize(s));
        need((e & 1) == 0, "b2g_assemble_pressure: a boundary face cell is outside [0, nCells)");
        need((e & 2) == 0, "b2g_assemble_pressure: a boundary type is not 0 (zeroGradient), 1 (fixedValue) or 2 (empty)");
        // each cell's boundary faces in patch-then-face order: a stable sort of the face indices by cell
        b2g::DBuf<int> bStart, bOrder, iota;
        b2g::DBuf<unsigned> keys;
        bStart.alloc(static_cast<size_t>(nC) + 1, s);
        b2g::countingStarts(bcell.p, nBFaces, nC, bStart.p, s);
        bOrder.alloc(std::max(nBFaces, 1), s);
        iota.alloc(std::max(nBFaces, 1), s);
        keys.alloc(std::max(nBFaces, 1), s);
        if (nBFaces) kAsmIota<<<blocks(nBFaces), 256, 0, s>>>(nBFaces, iota.p);
        int bits = 1;
        while ((1LL << bits) < nC) ++bits;
        b2g::sortPairs(reinterpret_cast<const unsigned*>(bcell.p), keys.p, iota.p, bOrder.p, nBFaces, bits, s);
        b2g::DBuf<double> dg, cf, src, ic, bc;
        dg.alloc(std::max(nC, 1), s);
        cf.alloc(std::max(nF, 1), s);
        src.alloc(std::max(nC, 1), s);
        ic.alloc(std::max(nBFaces, 1), s);
        bc.alloc(std::max(nBFaces, 1), s);
        if (nF) kAsmFaces<<<blocks(nF), 256, 0, s>>>(nF, L.lower.p, L.upper.p, w.p, dc.p, ms.p, rau.p, cf.p);
        if (nBFaces)
            kAsmBoundary<<<blocks(nBFaces), 256, 0, s>>>(nBFaces, bcell.p, rau.p, bms.p, bdc.p, btype.p, bval.p, ic.p,
                                                        bc.p);
        if (nC)
            kAsmCells<<<blocks(nC), 256, 0, s>>>(nC, L.rowStart.p, L.entFace.p, L.lower.p, cf.p, phi.p, bStart.p,
                                                 bOrder.p, btype.p, bphi.p, vol.p, dg.p, src.p);
        if (pRefCell >= 0) kAsmReference<<<1, 1, 0, s>>>(pRefCell, pRefValue, dg.p, src.p);
        B2G_LAUNCH_CHECK();
        const cudaMemcpyKind back = memspace == B2G_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        if (nC)
        {
            B2G_CUDA(cudaMemcpyAsync(diag, dg.p, sizeof(double) * nC, back, s));
            B2G_CUDA(cudaMemcpyAsync(source, src.p, sizeof(double) * nC, back, s));
        }
        if (nF) B2G_CUDA(cudaMemcpyAsync(upper, cf.p, sizeof(double) * nF, back, s));
        if (nBFaces)
        {
            B2G_CUDA(cudaMemcpyAsync(internalCoeffs, ic.p, sizeof(double) * nBFaces, back, s));
            B2G_CUDA(cudaMemcpyAsync(boundaryCoeffs, bc.p, sizeof(double) * nBFaces, back, s));
        }
        B2G_CUDA(cudaStreamSynchronize(s));
    });
}
