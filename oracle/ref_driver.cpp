// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY. An extern "C" shim, written for this repository, over
// the reference's OWN host implementation of the GAMG-PCG path. oracle/Makefile compiles it together
// with the reference's source files where they lie (nothing is copied) into oracle/_ref/libref.so.
// tests/ use it to pin oracle/gamg_oracle.c bit-for-bit, and bench.py's reference arm times it.
//
// Reference entry points driven (paths relative to the reference project root):
//   faceAreaPairGamgAgglomeration  src/matrices/lduMatrix/solvers/GAMG/GAMGAgglomerations/
//                                  pair_gamg_agglomeration_cpp.cuh:99-105
//   pcgGamgSolve (hierarchy form)  src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cuh:202-213
//   gamgSolveFolded                gamg_solver_cpp.cuh:185-192
//   gamgSolve (with patches)       gamg_solver_cpp.cuh:170-177 (one coupled patch: the pair)
//   gamgCoarsestPcgDic             gamg_solver_cpp.cuh:152-162
//   gaussSeidelSmoothFolded        src/OpenFOAM/matrices/smooth_solver_cpp.cuh
//   lduOwnerStart                  src/OpenFOAM/matrices/smooth_solver_cpp.cu:10-34
#include "gamg_solver_cpp.cuh"
#include "smooth_solver_cpp.cuh"
#include "fv_geometry.cuh"
#include "fv_patch.cuh"
#include "primitive_mesh.cuh"

#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace brae;

namespace {

std::string g_err;

struct RefAgglom
{
    GamgAgglomeration a;
};

const char* smootherName(int k)
{
    switch (k)
    {
        case 0: return "GaussSeidel";
        case 1: return "symGaussSeidel";
        case 2: return "DIC";
        case 3: return "DICGaussSeidel";
        default: return "unknown";
    }
}

// the layout of oc_controls in gamg_oracle.h
struct Controls
{
    int smoother;
    double tolerance;
    double relTol;
    int maxIter;
    int minIter;
    int nPreSweeps;
    int preSweepsLevelMultiplier;
    int maxPreSweeps;
    int nPostSweeps;
    int postSweepsLevelMultiplier;
    int maxPostSweeps;
    int nFinestSweeps;
    int scaleCorrection;
    int nCellsInCoarsestLevel;
    int nVcycles;
};

struct Perf
{
    double initialResidual;
    double finalResidual;
    int nIterations;
};

GamgControls toGamg(const Controls& c)
{
    GamgControls g;
    g.smoother = smootherName(c.smoother);
    g.tolerance = c.tolerance;
    g.relTol = c.relTol;
    g.maxIter = c.maxIter;
    g.minIter = c.minIter;
    g.nPreSweeps = c.nPreSweeps;
    g.preSweepsLevelMultiplier = c.preSweepsLevelMultiplier;
    g.maxPreSweeps = c.maxPreSweeps;
    g.nPostSweeps = c.nPostSweeps;
    g.postSweepsLevelMultiplier = c.postSweepsLevelMultiplier;
    g.maxPostSweeps = c.maxPostSweeps;
    g.nFinestSweeps = c.nFinestSweeps;
    g.scaleCorrection = c.scaleCorrection != 0;
    g.nCellsInCoarsestLevel = c.nCellsInCoarsestLevel;
    return g;
}

Perf toPerf(const SolverPerformance& p)
{
    return Perf{p.initialResidual, p.finalResidual, p.nIterations};
}

// A PrimitiveMesh that carries only what the path reads: nCells and the internal faces' owner and
// neighbour (no points, no boundary faces).
PrimitiveMesh addressingMesh(int nC, int nF, const int* lower, const int* upper)
{
    PrimitiveMesh m;
    m.assign({}, {}, std::vector<label>(1, 0), std::vector<label>(lower, lower + nF),
             std::vector<label>(upper, upper + nF), {}, nC);
    return m;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_agglomerate(int nC, int nF, const int* lower, const int* upper, const double* Sf,
                      const double* magSf, int nCoarsest, int* forward)
{
    try
    {
        PrimitiveMesh m = addressingMesh(nC, nF, lower, upper);
        FvGeometry g;
        FvGeometry::Built b;
        b.Cf.assign(static_cast<std::size_t>(nF), vector{0, 0, 0});
        b.Sf.resize(static_cast<std::size_t>(nF));
        for (int f = 0; f < nF; ++f)
        {
            b.Sf[static_cast<std::size_t>(f)] = vector{Sf[3 * f], Sf[3 * f + 1], Sf[3 * f + 2]};
        }
        b.magSf.assign(magSf, magSf + nF);
        b.C.assign(static_cast<std::size_t>(nC), vector{0, 0, 0});
        b.V.assign(static_cast<std::size_t>(nC), 1.0);
        b.weights.assign(static_cast<std::size_t>(nF), 0.5);
        b.deltaCoeffs.assign(static_cast<std::size_t>(nF), 1.0);
        b.nonOrthDeltaCoeffs.assign(static_cast<std::size_t>(nF), 1.0);
        b.nonOrthCorr.assign(static_cast<std::size_t>(nF), vector{0, 0, 0});
        g.adopt(b, m);
        bool fw = *forward != 0;
        RefAgglom* r = new RefAgglom;
        r->a = faceAreaPairGamgAgglomeration(m, g, nCoarsest, fw);
        *forward = fw ? 1 : 0;
        return r;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return nullptr;
    }
}

void ref_agglom_free(void* h) { delete static_cast<RefAgglom*>(h); }

int ref_agglom_nlevels(void* h) { return static_cast<RefAgglom*>(h)->a.size(); }

void ref_agglom_level_size(void* h, int level, int* nC, int* nF)
{
    const GamgLduAddressing& m = static_cast<RefAgglom*>(h)->a.meshLevel(level);
    *nC = m.nCells;
    *nF = static_cast<int>(m.upperAddr.size());
}

void ref_agglom_get(void* h, int step, int* restrictAddr, int* faceRestrict, char* flip,
                    int* coarseLower, int* coarseUpper)
{
    const GamgAgglomeration& a = static_cast<RefAgglom*>(h)->a;
    const std::size_t s = static_cast<std::size_t>(step);
    std::memcpy(restrictAddr, a.restrictAddressing[s].data(), sizeof(int) * a.restrictAddressing[s].size());
    std::memcpy(faceRestrict, a.faceRestrictAddressing[s].data(),
                sizeof(int) * a.faceRestrictAddressing[s].size());
    std::memcpy(flip, a.faceFlipMap[s].data(), a.faceFlipMap[s].size());
    std::memcpy(coarseLower, a.meshLevels[s].lowerAddr.data(), sizeof(int) * a.meshLevels[s].lowerAddr.size());
    std::memcpy(coarseUpper, a.meshLevels[s].upperAddr.data(), sizeof(int) * a.meshLevels[s].upperAddr.size());
}

// pcgGamgSolve on a folded system (no patches): returns 0 on success, -1 on a refusal
int ref_pcg_gamg_solve(void* h, const double* diag, const double* upper, const double* source,
                       double* psi, double tol, double relTol, int maxIter, int minIter,
                       const Controls* c, Perf* out, Perf* coarsest, int coarsestCap, int* nCoarsest)
{
    try
    {
        const GamgAgglomeration& a = static_cast<RefAgglom*>(h)->a;
        const int nC = a.fineMesh.nCells;
        const int nF = static_cast<int>(a.fineMesh.upperAddr.size());
        PrimitiveMesh m = addressingMesh(nC, nF, a.fineMesh.lowerAddr.data(), a.fineMesh.upperAddr.data());
        FvScalarMatrix M;
        M.diag.assign(diag, diag + nC);
        M.upper.assign(upper, upper + nF);
        M.lower = M.upper;
        M.source.assign(source, source + nC);
        std::vector<scalar> x(psi, psi + nC);
        GamgPreconditionerControls pc;
        pc.gamg = toGamg(*c);
        pc.nVcycles = c->nVcycles;
        GamgSolveLog log;
        const SolverPerformance p =
            pcgGamgSolve(M, x, m, {}, a, tol, relTol, maxIter, minIter, pc, &log);
        std::memcpy(psi, x.data(), sizeof(double) * static_cast<std::size_t>(nC));
        *out = toPerf(p);
        if (nCoarsest) *nCoarsest = static_cast<int>(log.coarsest.size());
        for (std::size_t i = 0; i < log.coarsest.size() && static_cast<int>(i) < coarsestCap; ++i)
        {
            coarsest[i] = toPerf(log.coarsest[i]);
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

int ref_gamg_solve(void* h, const double* diag, const double* upper, const double* source,
                   double* psi, const Controls* c, Perf* out)
{
    try
    {
        const GamgAgglomeration& a = static_cast<RefAgglom*>(h)->a;
        const int nC = a.fineMesh.nCells;
        const int nF = static_cast<int>(a.fineMesh.upperAddr.size());
        std::vector<scalar> d(diag, diag + nC), u(upper, upper + nF), s(source, source + nC);
        std::vector<scalar> x(psi, psi + nC);
        const SolverPerformance p = gamgSolveFolded(a, d, u, s, x, toGamg(*c), nullptr);
        std::memcpy(psi, x.data(), sizeof(double) * static_cast<std::size_t>(nC));
        *out = toPerf(p);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

// gamgSolve on a folded system plus one coupled patch carrying the pair: faceCells `own`, the
// neighbour cells `nbr` face for face, boundaryCoeffs `coeff` (the interface coefficients) and
// internalCoeffs zero, so foldBoundary leaves diag and source as they are handed in.
int ref_gamg_solve_pair(void* h, const double* diag, const double* upper, const double* source,
                        double* psi, int nIf, const int* own, const int* nbr, const double* coeff,
                        const Controls* c, Perf* out)
{
    try
    {
        const GamgAgglomeration& a = static_cast<RefAgglom*>(h)->a;
        const int nC = a.fineMesh.nCells;
        const int nF = static_cast<int>(a.fineMesh.upperAddr.size());
        PrimitiveMesh m = addressingMesh(nC, nF, a.fineMesh.lowerAddr.data(), a.fineMesh.upperAddr.data());
        FvScalarMatrix M;
        M.diag.assign(diag, diag + nC);
        M.upper.assign(upper, upper + nF);
        M.lower = M.upper;
        M.source.assign(source, source + nC);
        std::vector<FvPatch> patches(1);
        FvPatch& p = patches[0];
        p.name = "pair";
        p.type = "cyclic";
        p.size = nIf;
        p.faceCells.assign(own, own + nIf);
        p.nbrFaceCells.assign(nbr, nbr + nIf);
        p.coupled = true;
        M.internalCoeffs.assign(1, std::vector<scalar>(static_cast<std::size_t>(nIf), scalar(0)));
        M.boundaryCoeffs.assign(1, std::vector<scalar>(coeff, coeff + nIf));
        std::vector<scalar> x(psi, psi + nC);
        const SolverPerformance perf = gamgSolve(M, x, m, patches, a, toGamg(*c), nullptr);
        std::memcpy(psi, x.data(), sizeof(double) * static_cast<std::size_t>(nC));
        *out = toPerf(perf);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

int ref_gs_smooth(int nC, int nF, const int* lower, const int* upper, const double* diag,
                  const double* coef, double* psi, const double* b, int nSweeps, int symmetric)
{
    try
    {
        std::vector<label> lo(lower, lower + nF), up(upper, upper + nF);
        const std::vector<label> os = lduOwnerStart(lo, up, nC);
        std::vector<scalar> d(diag, diag + nC), c(coef, coef + nF), bb(b, b + nC), x(psi, psi + nC);
        gaussSeidelSmoothFolded(os, up, d, c, c, bb, x, nSweeps, symmetric != 0);
        std::memcpy(psi, x.data(), sizeof(double) * static_cast<std::size_t>(nC));
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

int ref_coarsest_pcg_dic(int nC, int nF, const int* lower, const int* upper, const double* diag,
                         const double* coef, double* psi, const double* source, double tol,
                         double relTol, Perf* out)
{
    try
    {
        GamgLduAddressing addr;
        addr.nCells = nC;
        addr.lowerAddr.assign(lower, lower + nF);
        addr.upperAddr.assign(upper, upper + nF);
        std::vector<scalar> d(diag, diag + nC), c(coef, coef + nF), s(source, source + nC), x(psi, psi + nC);
        const SolverPerformance p = gamgCoarsestPcgDic(addr, d, c, x, s, tol, relTol);
        std::memcpy(psi, x.data(), sizeof(double) * static_cast<std::size_t>(nC));
        *out = toPerf(p);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
