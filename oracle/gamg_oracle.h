/*
 * gamg_oracle.h -- TEST INFRASTRUCTURE ONLY. A plain-C restatement of the reference's host path
 * for the GAMG-preconditioned PCG pressure solve (simd-ai/brae), used by tests/, by smoke() and by
 * bench.py's CPU-baseline leg as the checker. Nothing in the product links, loads or calls it.
 *
 * Every function cites the reference file:line it restates. Paths are relative to the reference
 * project root:
 *   AGG  = src/matrices/lduMatrix/solvers/GAMG/GAMGAgglomerations/pair_gamg_agglomeration_cpp.cu
 *   GAMG = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu
 *   SMO  = src/OpenFOAM/matrices/smooth_solver_cpp.cu
 *
 * Parity is pinned two ways (tests/test_oracle_*.py): against the reference's own sources compiled
 * here into oracle/_ref (bit-for-bit: hierarchy, iteration count, residuals, solution), and against
 * OpenFOAM's dumped golden vectors from the reference's validation/ tree (tests/golden/).
 *
 * Build: gcc -O2 -ffp-contract=off (x86-64 without -march emits no FMA, matching the reference
 * built the same way). Types: label = int32, scalar = double.
 */
#ifndef GAMG_ORACLE_H
#define GAMG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GamgControls + GamgPreconditionerControls (gamg_solver_cpp.cuh:67-85, :128-132). */
typedef struct
{
    int smoother;           /* 0 GaussSeidel, 1 symGaussSeidel, 2 DIC, 3 DICGaussSeidel */
    double tolerance;       /* the GAMG entry's own (coarsest-level PCG uses it) */
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
} oc_controls;

typedef struct
{
    double initialResidual;
    double finalResidual;
    int nIterations;
} oc_perf;

typedef struct oc_agglom oc_agglom;

/* faceAreaPairGamgAgglomeration (AGG:286-345); `forward` is the static direction flag. */
oc_agglom* oc_agglomerate(int nCells, int nFaces, const int* lower, const int* upper,
                          const double* Sf, const double* magSf, int nCellsInCoarsestLevel,
                          int* forward);
void oc_agglom_free(oc_agglom* a);
int oc_agglom_nlevels(const oc_agglom* a);
/* sizes of coarse level i (i = 1..nLevels; level 0 is the mesh) */
void oc_agglom_level_size(const oc_agglom* a, int level, int* nCells, int* nFaces);
/* step i -> i+1 (i = 0..nLevels-1): restrictAddressing (nCells of level i), faceRestrictAddressing
 * and faceFlipMap (nFaces of level i); coarse addressing of level i+1 */
void oc_agglom_get(const oc_agglom* a, int step, int* restrictAddr, int* faceRestrict,
                   char* flip, int* coarseLower, int* coarseUpper);
/* the weights the pairing pass of step i compared (nFaces of level i) */
void oc_agglom_weights(const oc_agglom* a, int step, double* w);

/* Galerkin coarse matrices (GAMG:474-526); level i = 1..nLevels */
typedef struct oc_hier oc_hier;
oc_hier* oc_hier_build(const oc_agglom* a, const double* diag, const double* upper);
/* ... with the finest level's coupled pair (nIf faces, each once from its own side; ifCoeff in the
 * sign convention Amul subtracts, GAMG:25-36) and every coarse level's agglomerated from it
 * (GAMG:497-524) */
oc_hier* oc_hier_build_pair(const oc_agglom* a, const double* diag, const double* upper, int nIf,
                            const int* ifOwn, const int* ifNbr, const double* ifCoeff);
void oc_hier_free(oc_hier* h);
void oc_hier_level(const oc_hier* h, int level, double* diag, double* upper);
/* level `level`'s pair (any array may be NULL); returns its face count */
int oc_hier_level_pair(const oc_hier* h, int level, int* ifOwn, int* ifNbr, double* ifCoeff);

/* lduMatrix pieces on one level (GAMG:62-191) */
void oc_amul(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
             const double* coef, const double* psi, double* Apsi);
double oc_norm_factor(int nCells, int nFaces, const int* lower, const int* upper,
                      const double* diag, const double* coef, const double* psi,
                      const double* source, const double* Apsi);
double oc_sum_mag(int n, const double* x);
double oc_sum_prod(int n, const double* a, const double* b);

/* smoothers (GAMG:234-317, SMO:87-166) */
void oc_smooth(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
               const double* coef, double* psi, const double* source, int nSweeps, int smoother);

/* coarsest PCG-DIC (GAMG:321-383), from the psi handed in */
oc_perf oc_pcg_dic(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
                   const double* coef, double* psi, const double* source, double tolerance,
                   double relTol, int maxIter);

/* GAMG::scale (GAMG:386-407) */
void oc_scale(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
              const double* coef, double* field, double* Acf, const double* source);

/* GAMGPreconditioner::precondition: w = M^-1 r with nVcycles V-cycles from zero (GAMG:1089-1107).
 * Coarsest-level performances are appended to `coarsest` (capacity `cap`, count in *nCoarsest). */
void oc_precondition(const oc_hier* h, const oc_controls* c, double* w, const double* r,
                     oc_perf* coarsest, int cap, int* nCoarsest);

/* pcgGamgSolveImpl (GAMG:1031-1143) on a folded system. `history` (capacity cap) receives the
 * residual after each PCG iteration; `coarsest` the coarsest-level performances of every V-cycle. */
oc_perf oc_pcg_gamg_solve(const oc_agglom* a, const double* diag, const double* upper,
                          const double* source, double* psi, double tolerance, double relTol,
                          int maxIter, int minIter, const oc_controls* c, double* history,
                          int historyCap, oc_perf* coarsest, int coarsestCap, int* nCoarsest);

/* gamgSolveFoldedImpl (GAMG:961-1027): the standalone GAMG solver */
oc_perf oc_gamg_solve(const oc_agglom* a, const double* diag, const double* upper,
                      const double* source, double* psi, const oc_controls* c, double* history,
                      int historyCap);
/* gamgSolve with a coupled patch (GAMG:943-959): the same on a folded system with the finest
 * level's pair (as oc_hier_build_pair takes it) */
oc_perf oc_gamg_solve_pair(const oc_agglom* a, const double* diag, const double* upper, int nIf,
                           const int* ifOwn, const int* ifNbr, const double* ifCoeff,
                           const double* source, double* psi, const oc_controls* c, double* history,
                           int historyCap);
/* Amul and Smoother::smooth on one level with a pair (GAMG:82-87, :287-305) */
void oc_amul_pair(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
                  const double* coef, int nIf, const int* ifOwn, const int* ifNbr, const double* ifCoeff,
                  const double* psi, double* Apsi);
void oc_smooth_pair(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
                    const double* coef, int nIf, const int* ifOwn, const int* ifNbr, const double* ifCoeff,
                    double* psi, const double* source, int nSweeps, int smoother);

/* The pressure equation's assembly before the solve (simpleFoam pEqn.H stages 4-5, the reference's
 * cpu::assemblePEqn, src/applications/solvers/simpleFoam/pEqn_cpp.cu:209-260) on an orthogonal mesh
 * with uncoupled patches: fvc::interpolate(rAU) (fvc.cu:626-650; a boundary face takes its cell's
 * value), fvm::laplacian (fvm.cuh:130-150: upper = lower = deltaCoeffs*rAUf*|Sf| per internal face,
 * diag = minus their sum in face order; laplacianBoundaryCoeffs fvm.cuh:40-95 with the fixedValue
 * gradient coefficients fv_patch_field.cuh:590-602, zeroGradient's zero), source = div(phiHbyA)*V
 * (fvc.cu:706-730: the face sum in face order, the boundary faces patch by patch, divided by V, then
 * multiplied by V back), and setReference (pEqn_cpp.cu:248-255). Boundary faces are given patch by
 * patch: bType 1 fixedValue bValue, 0 zeroGradient, 2 empty (left out of the divergence). */
void oc_assemble_pressure(int nCells, int nFaces, const int* lower, const int* upper, const double* weights,
                          const double* deltaCoeffs, const double* magSf, const double* V, const double* rAU,
                          const double* phi, int nBFaces, const int* bFaceCells, const double* bMagSf,
                          const double* bDeltaCoeffs, const int* bType, const double* bValue,
                          const double* bPhi, int pRefCell, double pRefValue, double* diag, double* coef,
                          double* source, double* internalCoeffs, double* boundaryCoeffs);

#ifdef __cplusplus
}
#endif

#endif
