// ref_peqn.cpp -- TEST INFRASTRUCTURE ONLY. An extern "C" shim, written for this repository, over the
// reference's OWN assembly of the pressure equation (simpleFoam's pEqn.H stage 4-5), compiled with the
// reference's sources where they lie (oracle/Makefile; nothing is copied) into oracle/_ref/libref.so.
// tests/ use it to pin oracle/gamg_oracle.c's restatement and the device assembly bit for bit.
//
// Reference entry points driven (paths relative to the reference project root):
//   cpu::assemblePEqn          src/applications/solvers/simpleFoam/pEqn_cpp.cu:209-260
//   boxtest::boxMesh           tests/box_mesh.cuh (the reference's own in-memory hex box: internal faces
//                              upper-triangular, then patches inlet, outlet, wallYmin, wallYmax,
//                              wallZmin, wallZmax)
//   FvGeometry::build, buildPatches, buildField (the geometry and the pressure field's patches)
#include "box_mesh.cuh"
#include "geometric_field.cuh"
#include "pEqn_cpp.cuh"

#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace brae;

namespace {
std::string g_peqnErr;

template <class T>
void put(const std::vector<T>& v, T* out)
{
    if (out && !v.empty()) std::memcpy(out, v.data(), sizeof(T) * v.size());
}
}  // namespace

extern "C" {

const char* ref_peqn_last_error() { return g_peqnErr.c_str(); }

// The orthogonal box Nx x Ny x Nz with cell sizes dx, dy, dz; per patch (the order above) the pressure
// condition: patchFixed[i] 1 for fixedValue patchValue[i], 0 for zeroGradient. Inputs rAU [nCells],
// phiHbyA on the internal faces [nInternalFaces] and on the boundary faces [nBoundaryFaces, patch by
// patch]; pRefCell -1 for none. Outputs (any may be null): the geometry the assembly read (face
// addressing, weights, deltaCoeffs, |Sf|, V; per boundary face its cell, |Sf| and deltaCoeffs), and the
// assembled matrix: diag [nCells], upper [nInternalFaces] (lower == upper), source [nCells], per boundary
// face internalCoeffs and boundaryCoeffs.
int ref_box_assemble_peqn(int Nx, int Ny, int Nz, double dx, double dy, double dz, const int* patchFixed,
                          const double* patchValue, const double* rAU, const double* phiInternal,
                          const double* phiBoundary, int pRefCell, double pRefValue, int* lower, int* upper,
                          double* weights, double* deltaCoeffs, double* magSf, double* V, int* bFaceCells,
                          double* bMagSf, double* bDeltaCoeffs, double* diag, double* upperCoef, double* source,
                          double* internalCoeffs, double* boundaryCoeffs)
{
    try
    {
        const PrimitiveMesh m = boxtest::boxMesh(Nx, Ny, Nz, 0.0, dx, dy, dz);
        FvGeometry g;
        g.build(m);
        const std::vector<FvPatch> patches = buildPatches(m, g);
        const label nC = m.nCells();
        const label nIf = m.nInternalFaces();
        FieldData<scalar> fd;
        fd.internalUniform = true;
        fd.internalUniformValue = 0.0;
        for (std::size_t pi = 0; pi < patches.size(); ++pi)
        {
            const bool fixed = patchFixed[pi] != 0;
            fd.boundary.push_back(boxtest::pfd<scalar>(patches[pi].name.c_str(), fixed ? "fixedValue" : "zeroGradient",
                                                       fixed ? patchValue[pi] : 0.0, fixed));
        }
        GeometricField<scalar> p = buildField<scalar>(fd, patches, nC);
        p.evaluateBoundary();
        cpu::PressureStages st;
        st.rAU.assign(rAU, rAU + nC);
        st.rAtU = st.rAU;
        st.phiHbyA.internal.assign(phiInternal, phiInternal + nIf);
        st.phiHbyA.boundary.resize(patches.size());
        std::size_t b = 0;
        for (std::size_t pi = 0; pi < patches.size(); ++pi)
        {
            st.phiHbyA.boundary[pi].assign(phiBoundary + b, phiBoundary + b + patches[pi].size);
            b += static_cast<std::size_t>(patches[pi].size);
        }
        cpu::PressureInput in;
        in.pRefCell = pRefCell;
        in.pRefValue = pRefValue;
        const FvScalarMatrix M = cpu::assemblePEqn(st, p, in, m, g, patches);
        if (lower) std::memcpy(lower, m.owner().data(), sizeof(int) * static_cast<std::size_t>(nIf));
        if (upper) std::memcpy(upper, m.neighbour().data(), sizeof(int) * static_cast<std::size_t>(nIf));
        if (weights) std::memcpy(weights, g.weights().data(), sizeof(double) * static_cast<std::size_t>(nIf));
        if (deltaCoeffs) std::memcpy(deltaCoeffs, g.deltaCoeffs().data(), sizeof(double) * static_cast<std::size_t>(nIf));
        if (magSf) std::memcpy(magSf, g.magSf().data(), sizeof(double) * static_cast<std::size_t>(nIf));
        put(g.V(), V);
        put(M.diag, diag);
        put(M.upper, upperCoef);
        put(M.source, source);
        b = 0;
        for (std::size_t pi = 0; pi < patches.size(); ++pi)
        {
            const FvPatch& fp = patches[pi];
            for (label i = 0; i < fp.size; ++i, ++b)
            {
                if (bFaceCells) bFaceCells[b] = fp.faceCells[i];
                if (bMagSf) bMagSf[b] = fp.magSf[i];
                if (bDeltaCoeffs) bDeltaCoeffs[b] = fp.deltaCoeffs[i];
                if (internalCoeffs) internalCoeffs[b] = M.internalCoeffs[pi][i];
                if (boundaryCoeffs) boundaryCoeffs[b] = M.boundaryCoeffs[pi][i];
            }
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_peqnErr = e.what();
        return -1;
    }
}

}  // extern "C"
