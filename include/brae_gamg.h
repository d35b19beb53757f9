/*
 * brae_gamg.h -- C ABI of the B200-native GAMG-preconditioned PCG pressure solver.
 *
 * A drop-in for the reference's (simd-ai/brae) pressure linear solve: OpenFOAM's PCG with the GAMG
 * preconditioner on a symmetric LDU matrix -- faceAreaPair agglomeration, GaussSeidel smoothing,
 * restriction/prolongation, the coarsest-level PCG-DIC, lduMatrix::Amul and the normFactor / dot
 * reductions -- all on one GPU. Plain pointers and sizes only; no C++ or torch types cross it.
 *
 * Citations name the reference interface each entry point replaces (paths relative to the
 * reference project root):
 *   GAMGH = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cuh
 *   AGGH  = src/matrices/lduMatrix/solvers/GAMG/GAMGAgglomerations/pair_gamg_agglomeration_cpp.cuh
 *   DGAMG = src/matrices/lduMatrix/solvers/GAMG/device_gamg_solver.cuh
 *   GAMG  = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu
 *   DGAMGC = src/matrices/lduMatrix/solvers/GAMG/device_gamg_solver.cu
 *   PCGH  = src/OpenFOAM/matrices/pcg.cuh
 *
 * Conventions
 *   - label = int32, scalar = double. The LDU addressing is OpenFOAM's: `lower` (owner) and
 *     `upper` (neighbour) per internal face, faces sorted by owner, owner < neighbour.
 *   - The matrix is the FOLDED symmetric system the solver receives (boundary internalCoeffs in
 *     `diag`, boundaryCoeffs in `source`), as gamgSolveFolded takes it (GAMGH:185-192).
 *   - `memspace` says where array arguments live: B2G_MEM_HOST (pageable or pinned host memory;
 *     copies are made on the stream) or B2G_MEM_DEVICE (device pointers on the current device).
 *   - `stream` is a cudaStream_t; NULL means cudaStreamPerThread, the reference's stream
 *     (cmake/BraeCompilerOptions.cmake:9-12). Calls return after the work they describe is
 *     complete unless stated otherwise.
 *   - Every call returns a b2g_status; on failure b2g_last_error() gives a message naming the
 *     refused input, as the reference's std::runtime_error messages do (gamg_solver_cpp.cu:737-766).
 *   - Handles are not re-entrant: one host thread at a time per handle.
 */
#ifndef BRAE_GAMG_H
#define BRAE_GAMG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2G_API __attribute__((visibility("default")))

typedef enum
{
    B2G_OK = 0,
    B2G_ERR_ARGUMENT = 1,        /* malformed input: sizes, null pointers, addressing order */
    B2G_ERR_REFUSED = 2,         /* an input the reference refuses by name (gamg_solver_cpp.cu:801-928) */
    B2G_ERR_CUDA = 3,            /* a CUDA runtime error */
    B2G_ERR_NO_MEMORY = 4,       /* device allocation failed, or a request exceeds an admission cap */
    B2G_ERR_DEVICE_TIMEOUT = 5,  /* a bounded device-side wait gave up; the result is invalid */
    B2G_ERR_STATE = 6            /* a handle used out of order */
} b2g_status;

enum
{
    B2G_MEM_HOST = 0,
    B2G_MEM_DEVICE = 1
};

/* lduMatrix::smoother::New on a symmetric matrix, as GAMGSolver selects it (gamgSmootherPorted,
 * GAMGH:136) */
enum
{
    B2G_SMOOTHER_GAUSS_SEIDEL = 0,
    B2G_SMOOTHER_SYM_GAUSS_SEIDEL = 1,
    B2G_SMOOTHER_DIC = 2,
    B2G_SMOOTHER_DIC_GAUSS_SEIDEL = 3
};

enum
{
    B2G_PRECISION_FP64 = 0,        /* the parity form: everything in FP64 */
    B2G_PRECISION_FP32_PRECOND = 1, /* FP64 outer PCG, FP32 V-cycle, flexible (Polak-Ribiere) beta */
    /* The same, with the FP32 V-cycle's Gauss-Seidel sweeps taken colour by colour: a greedy
     * colouring of each level (two colours on a structured hex level) whose cells of one colour
     * share no face, each colour one parallel update of its cells. The same GaussSeidel update in
     * another cell order; bandwidth-bound where the sequential order is bound by the sweep's
     * dependency chain. Built on first use (a greedy colouring by sweep depth, on the device). */
    B2G_PRECISION_FP32_PRECOND_MULTICOLOUR = 2
};

/* How sums and dot products are reduced. TREE is a fixed-shape parallel tree (deterministic, fast);
 * SERIAL adds in the reference's own order, one term after another (gamg_solver_cpp.cu:119-181), so
 * the whole FP64 solve is bit-identical to the reference's host path -- a verification mode whose
 * reductions cost n dependent additions each. */
enum
{
    B2G_REDUCTION_TREE = 0,
    B2G_REDUCTION_SERIAL = 1
};

/* The solver entry's controls: PCG's tolerance/relTol/maxIter/minIter (lduMatrixSolver.C:195-205
 * via inter_case_cpp.cu:1519-1572) and the `preconditioner { preconditioner GAMG; ... }`
 * sub-dictionary's GamgControls + nVcycles (GAMGH:67-85, :128-132). Defaults: b2g_controls_default. */
enum
{
    B2G_SOLVER_PCG_GAMG = 0,       /* solver PCG; preconditioner { preconditioner GAMG; ... } */
    B2G_SOLVER_GAMG = 1            /* solver GAMG; (the standalone GAMGSolver) */
};

typedef struct
{
    int solver;                  /* B2G_SOLVER_PCG_GAMG */
    /* PCG (the solver entry); for solver GAMG, the GAMG entry's own */
    double tolerance;            /* 1e-6 */
    double relTol;               /* 0 */
    int maxIter;                 /* 1000 */
    int minIter;                 /* 0 */
    /* GAMG preconditioner (its own dictionary) */
    int smoother;                /* mandatory in the dictionary; GaussSeidel here */
    double precTolerance;        /* 1e-6: the coarsest-level PCG-DIC stops on these two */
    double precRelTol;           /* 0 */
    int nPreSweeps;              /* 0 */
    int preSweepsLevelMultiplier;/* 1 */
    int maxPreSweeps;            /* 4 */
    int nPostSweeps;             /* 2 */
    int postSweepsLevelMultiplier;/* 1 */
    int maxPostSweeps;           /* 4 */
    int nFinestSweeps;           /* 2 */
    int scaleCorrection;         /* 1 (the matrix is symmetric) */
    int nCellsInCoarsestLevel;   /* 10 */
    int nVcycles;                /* 2 (GAMGPreconditioner.C:60) */
    int precision;               /* B2G_PRECISION_FP64 */
    int reduction;               /* B2G_REDUCTION_TREE */
    /* 1: the FP32-preconditioned forms solve the coarsest level directly, by a dense FP64 Cholesky
     * factor made once per coarse matrix (up to 96 cells; a level that is not positive definite
     * keeps PCG-DIC), as the reference's precision form does; 0: PCG-DIC to precTolerance /
     * precRelTol. The FP64 form always runs the reference's PCG-DIC. No fvSolution key. */
    int coarsestDirect;          /* 1 */
} b2g_controls;

/* SolverPerformance (PCGH:16-21) */
typedef struct
{
    double initialResidual;
    double finalResidual;
    int nIterations;
} b2g_perf;

/* Optional per-solve record. `history[k]` = the normalised residual after PCG iteration k;
 * `coarsest` = the coarsest-level PCG-DIC performance of every V-cycle, as GamgSolveLog holds it
 * (GAMGH:147-150). The caller owns the arrays and states their capacities; counts are written back
 * (they may exceed the capacities, in which case only the first entries are stored). */
typedef struct
{
    double* history;
    int historyCapacity;
    int historyCount;
    b2g_perf* coarsest;
    int coarsestCapacity;
    int coarsestCount;
} b2g_solve_log;

typedef struct b2g_mesh b2g_mesh;     /* a mesh's GAMG hierarchy (GamgAgglomerationCache) */
typedef struct b2g_matrix b2g_matrix; /* one matrix on that hierarchy (GamgHierarchy) */

/* ---- errors and controls -------------------------------------------------------------------- */

/* The message of the last failed call on this thread ("" if none). */
B2G_API const char* b2g_last_error(void);

/* GAMGSolver.C's and lduMatrix::solver's defaults, with smoother GaussSeidel. */
B2G_API b2g_status b2g_controls_default(b2g_controls* out);

/* Reads one fvSolution solver entry -- the text between (and excluding) its braces, e.g.
 * "solver PCG; tolerance 1e-6; relTol 0; preconditioner { preconditioner GAMG; smoother
 * GaussSeidel; nCellsInCoarsestLevel 10; }" -- into controls, refusing by name every key the
 * reference refuses: a solver other than PCG, a preconditioner other than GAMG, an unported or
 * asymmetric-only smoother, agglomerator != faceAreaPair, mergeLevels != 1, updateInterval != 1,
 * cacheAgglomeration no, interpolateCorrection, directSolveCoarsest, a coarsestLevelCorr
 * sub-dictionary, processorAgglomerator. Replaces readGamgControls (GAMGH:139-144) and the PCG keys
 * of inter_case_cpp.cu:1519-1572. */
B2G_API b2g_status b2g_controls_read(const char* entryText, b2g_controls* out);

/* ---- the hierarchy (once per mesh) ---------------------------------------------------------- */

/* Builds the faceAreaPair agglomeration of a mesh on the device: face weights, the alternating
 * greedy pairing, the coarse addressing numbered owner-major by first appearance, face restrict
 * and flip maps, restricted weights -- bit-for-bit the reference's hierarchy.
 * Replaces faceAreaPairGamgAgglomeration (AGGH:99-105) behind GamgAgglomerationCache::get
 * (GAMGH:110-122) and its device upload DeviceGamgCache::get (DGAMG:109-127).
 * `Sf` is [nFaces][3], `magSf` [nFaces]. `forwardInOut` is the pairing direction flag OpenFOAM
 * keeps as a static (pairGAMGAgglomeration::forward_): read on entry, written back as the build
 * leaves it. Arrays are read from `memspace`; the handle keeps device copies. */
B2G_API b2g_status b2g_mesh_create(int nCells, int nFaces, const int32_t* lower,
                                   const int32_t* upper, const double* Sf, const double* magSf,
                                   int nCellsInCoarsestLevel, int* forwardInOut, int memspace,
                                   void* stream, b2g_mesh** out);
/* b2g_mesh_create with a hierarchy cache on disk (the warm start brae's own AMG cache gives,
 * device_amg_cache.cu): the agglomeration's inputs (sizes, lower, upper, Sf, magSf,
 * nCellsInCoarsestLevel, the direction flag) are hashed on the device; if `cachePath` holds an
 * agglomeration with the same signature its restriction maps are used and the pairing passes skipped
 * (*fromCache = 1, *forwardInOut set as the original build left it), else the hierarchy is built and
 * written there (*fromCache = 0). The hierarchy is the same either way. fromCache may be NULL. */
B2G_API b2g_status b2g_mesh_create_cached(int nCells, int nFaces, const int32_t* lower, const int32_t* upper,
                                          const double* Sf, const double* magSf, int nCellsInCoarsestLevel,
                                          int* forwardInOut, int memspace, void* stream, const char* cachePath,
                                          b2g_mesh** out, int* fromCache);
B2G_API b2g_status b2g_mesh_destroy(b2g_mesh* mesh);

/* Number of coarse levels (GamgAgglomeration::size(), AGGH:76-79). */
B2G_API b2g_status b2g_mesh_levels(const b2g_mesh* mesh, int* nLevels);
/* Cells and faces of level `level` (0 = the mesh, 1..nLevels = coarse levels). */
B2G_API b2g_status b2g_mesh_level_size(const b2g_mesh* mesh, int level, int* nCells,
                                       int* nFaces);
/* Copies step `step` (level step -> step+1) to HOST arrays, any of which may be NULL:
 * restrictAddressing [nCells(step)], faceRestrictAddressing [nFaces(step)], faceFlipMap
 * [nFaces(step)], coarse lower/upper [nFaces(step+1)] (AGGH:69-75). */
B2G_API b2g_status b2g_mesh_get_step(const b2g_mesh* mesh, int step, int32_t* restrictAddr,
                                     int32_t* faceRestrict, int8_t* flip, int32_t* coarseLower,
                                     int32_t* coarseUpper);
/* Milliseconds of device time the hierarchy build took (agglomeration plus the per-level
 * schedules), measured with events on the build stream. */
B2G_API b2g_status b2g_mesh_build_ms(const b2g_mesh* mesh, float* ms);

/* ---- the solve ------------------------------------------------------------------------------ */

/* PCG::scalarSolve with the GAMG preconditioner on a folded system: psi (initial guess honoured)
 * is overwritten with the solution; `out` receives the SolverPerformance. The preconditioner is
 * built only when the initial residual has not already converged (PCG.C:111-118).
 * Replaces pcgGamgSolve (GAMGH:217-229) and devicePcgGamgSolve (DGAMG:143-154).
 * `diag`, `source`, `psi` are [nCells], `upper` is [nFaces] (lower == upper). `log` may be NULL.
 * The mesh keeps the matrix it solves on between calls (its buffers and captured iteration graphs):
 * each call replaces its coefficients and rebuilds the coarse levels. Calls on one mesh must not
 * overlap (the reference's solve is not re-entrant either). */
B2G_API b2g_status b2g_pcg_gamg_solve(b2g_mesh* mesh, const double* diag, const double* upper,
                                      const double* source, double* psi,
                                      const b2g_controls* controls, int memspace, void* stream,
                                      b2g_perf* out, b2g_solve_log* log);

/* GAMGSolver::solve on a folded system: the standalone GAMG solver (V-cycles until converged).
 * Replaces gamgSolveFolded (GAMGH:185-192) and deviceGamgSolve. The GAMG tolerance, relTol,
 * maxIter and minIter are controls->tolerance/relTol/maxIter/minIter. */
B2G_API b2g_status b2g_gamg_solve(b2g_mesh* mesh, const double* diag, const double* upper,
                                  const double* source, double* psi,
                                  const b2g_controls* controls, int memspace, void* stream,
                                  b2g_perf* out, b2g_solve_log* log);

/* ---- the coupled (cyclic) pair ------------------------------------------------------------------ */

/* The mesh's coupled pair, once per mesh: the faces of its coupled (cyclic) patches, each once from
 * its own side -- faceCells[i] the cell the face belongs to, nbrFaceCells[i] the cell across the pair
 * -- in patch order, then face order, as gamgLevel0Interface lists them (GAMG:440-470). Every coarse
 * level's pair is agglomerated from it on the coarse cell pair, the first face of a pair making the
 * coarse face and later ones merging into it (agglomerateMatrix, GAMG:497-524; the reference's device
 * arm builds the same in buildGamgInterfaces, DGAMGC:335-391). A second call is refused. */
B2G_API b2g_status b2g_mesh_set_pair(b2g_mesh* mesh, int nPairFaces, const int32_t* faceCells,
                                     const int32_t* nbrFaceCells, int memspace, void* stream);
/* Level `level`'s pair: *nPairFaces and, if not NULL, its faces' cells (HOST arrays of that size). */
B2G_API b2g_status b2g_mesh_level_pair(const b2g_mesh* mesh, int level, int* nPairFaces, int32_t* own,
                                       int32_t* nbr);

/* gamgSolve with coupled patches (GAMGH:174-181; its device arm deviceGamgSolve, DGAMGC:713-764): the standalone GAMG solve of a folded system whose coupled patches carry the pair.
 * `pairCoeffs` [nPairFaces] are the coupled patches' boundaryCoeffs in b2g_mesh_set_pair's face
 * order, in the reference's sign convention: Amul subtracts pairCoeffs[i]*psi[nbrFaceCells[i]] from
 * row faceCells[i]. Their diagonal share (the patches' internalCoeffs) is folded into `diag`; their
 * source is not folded (b2g_fold_boundary with the coupled flag set). The pair enters the residual,
 * normFactor's row sums, every level's Amul, the Gauss-Seidel smoothers' bPrime once per smoothing
 * call, DIC through the residual, and the coarsest PCG-DIC (GAMG:82-145, :287-305). FP64 form only.
 * PCG with the GAMG preconditioner refuses a coupled matrix, as the reference's pcgGamgSolve does
 * (GAMG:1045). */
B2G_API b2g_status b2g_gamg_solve_coupled(b2g_mesh* mesh, const double* diag, const double* upper,
                                          const double* pairCoeffs, const double* source, double* psi,
                                          const b2g_controls* controls, int memspace, void* stream,
                                          b2g_perf* out, b2g_solve_log* log);
/* b2g_matrix_create with the pair's coefficients: every level's pair coefficient is restricted from
 * the finer level's (the sum from zero over the merged faces in ascending face order, GAMG:520-522)
 * and the level entries below (Amul, smoothing, scale, normFactor, the coarsest PCG-DIC) carry it. */
B2G_API b2g_status b2g_matrix_create_coupled(b2g_mesh* mesh, const double* diag, const double* upper,
                                             const double* pairCoeffs, int memspace, void* stream,
                                             b2g_matrix** out);
/* Level `level`'s pair coefficients (HOST array of b2g_mesh_level_pair's size). */
B2G_API b2g_status b2g_matrix_level_pair_coeffs(const b2g_matrix* m, int level, double* coeffs);
/* The standalone GAMG solve on an existing matrix (coupled or not), source and psi in `memspace`. */
B2G_API b2g_status b2g_matrix_gamg_solve(b2g_matrix* m, const double* source, double* psi,
                                         const b2g_controls* controls, int memspace, b2g_perf* out,
                                         b2g_solve_log* log);

/* ---- one matrix on the hierarchy: the pieces, for callers that drive them (and for tests) ---- */

/* GamgHierarchy::build (gamg_solver_cpp.cu:565-623): uploads the folded fine matrix and builds
 * every coarse matrix by Galerkin summation in the reference's order (agglomerateMatrix,
 * gamg_solver_cpp.cu:474-526), plus the per-level coefficient layouts the kernels read. */
B2G_API b2g_status b2g_matrix_create(b2g_mesh* mesh, const double* diag, const double* upper,
                                     int memspace, void* stream, b2g_matrix** out);
/* New coefficients for an existing matrix on the same mesh (the next time step's pressure matrix):
 * the fine level is replaced and every coarse level rebuilt, as GamgHierarchy::build does in each
 * pcgGamgSolve call (gamg_solver_cpp.cu:1081-1083), into the buffers the matrix already holds, so
 * its captured iteration graphs are replayed, not captured again. Refused for a coupled matrix. */
B2G_API b2g_status b2g_matrix_set_coeffs(b2g_matrix* m, const double* diag, const double* upper,
                                         int memspace);
B2G_API b2g_status b2g_matrix_destroy(b2g_matrix* m);
/* Copies level `level`'s diag [nCells] and upper [nFaces] to HOST arrays. */
B2G_API b2g_status b2g_matrix_get_level(const b2g_matrix* m, int level, double* diag,
                                        double* upper);

/* The following take DEVICE pointers sized for level `level` and run on the matrix's stream. */

/* lduMatrix::Amul (gamg_solver_cpp.cu:62-88): y = A x, bit-for-bit the reference's order. */
B2G_API b2g_status b2g_level_amul(b2g_matrix* m, int level, const double* x, double* y);
/* Smoother::smooth (gamg_solver_cpp.cu:262-316) with `smoother` B2G_SMOOTHER_*: nSweeps sweeps of
 * psi against source, in the sequential sweep order bit for bit. */
B2G_API b2g_status b2g_level_smooth(b2g_matrix* m, int level, int smoother, double* psi,
                                    const double* source, int nSweeps);
/* GAMGSolver::scale (gamg_solver_cpp.cu:386-407); Acf is scratch [nCells]. */
B2G_API b2g_status b2g_level_scale(b2g_matrix* m, int level, double* field, double* Acf,
                                   const double* source);
/* restrictField / prolongField across step `step` (gamg_solver_cpp.cu:410-432). */
B2G_API b2g_status b2g_step_restrict(b2g_matrix* m, int step, const double* fine, double* coarse);
B2G_API b2g_status b2g_step_prolong(b2g_matrix* m, int step, const double* coarse, double* fine);
/* lduMatrix::solver::normFactor (gamg_solver_cpp.cu:119-159), written to *nf (host). */
B2G_API b2g_status b2g_level_norm_factor(b2g_matrix* m, int level, const double* psi,
                                         const double* source, const double* Apsi, double* nf);
/* The coarsest-level PCG-DIC (gamg_solver_cpp.cu:321-383) on level `level` from psi. */
B2G_API b2g_status b2g_level_pcg_dic(b2g_matrix* m, int level, double* psi, const double* source,
                                     double tolerance, double relTol, b2g_perf* out);
/* b2g_level_pcg_dic without any device allocation: no counterpart in the reference. For callers that
 * may not allocate device memory during a solve (device memory owned by another allocator, or no
 * room for the synchronisation cudaMalloc/cudaFree can bring). Its scratch vectors live in one
 * static device array of the library (about 192 KiB, held on every GPU that loads the library until
 * the process exits), so levels of at most 4096 cells are accepted; larger ones return
 * B2G_ERR_ARGUMENT. The matrix's device must be current. The first call on a device looks the
 * array's device address up (make it before any stream capture). Every call shares the array:
 * calls that overlap on the GPU (other streams, other threads) race. Results are bit for bit those
 * of b2g_level_pcg_dic. */
B2G_API b2g_status b2g_level_pcg_dic_static(b2g_matrix* m, int level, double* psi, const double* source,
                                            double tolerance, double relTol, b2g_perf* out);
/* GAMGPreconditioner::precondition (gamg_solver_cpp.cu:1089-1107): w = M^-1 r, nVcycles V-cycles
 * from zero. `log` (may be NULL) receives the coarsest-level performances. */
B2G_API b2g_status b2g_precondition(b2g_matrix* m, const b2g_controls* controls, double* w,
                                    const double* r, b2g_solve_log* log);
/* The PCG solve on an existing matrix (the same as b2g_pcg_gamg_solve after b2g_matrix_create),
 * with source and psi in `memspace`. */
B2G_API b2g_status b2g_matrix_pcg_solve(b2g_matrix* m, const double* source, double* psi,
                                        const b2g_controls* controls, int memspace,
                                        b2g_perf* out, b2g_solve_log* log);

/* ---- introspection ---------------------------------------------------------------------------- */

/* Device time of the last solve on `m` by kernel class (milliseconds, `ms4`) and counts of each
 * class (`counts4`): [0] plain Amuls on the finest level (those fused with another step count as
 * everything else), [1] smoothing on the finest level (the count is sweeps), [2] everything else
 * (the count is launches), [3] the whole solve (all launches). Times
 * are taken with events on the solve's stream only while b2g_set_profiling(1) is on (the launch
 * count always). Either pointer may be NULL. */
B2G_API b2g_status b2g_matrix_timings(const b2g_matrix* m, double* ms4, long long* counts4);
/* The same per level, for `kind` 0 (Amul), 1 (smoothing calls) or 2 (Amul fused with another step:
 * the residual between V-cycles, the correction scaling's dots, the finest prolongation): for levels
 * 0..capacity-1, milliseconds, timed regions and units (Amuls, or the sweeps of the smoothing calls)
 * of the last solve. *nLevels receives the number of levels with a record. Any array may be NULL. */
B2G_API b2g_status b2g_matrix_level_timings(const b2g_matrix* m, int kind, int capacity, double* ms,
                                            long long* regions, long long* units, int* nLevels);
B2G_API b2g_status b2g_set_profiling(int on);
/* Whether the exact Gauss-Seidel smoothing calls may run all their sweeps in one pipelined launch
 * (on by default; the choice per level is made by measurement on a matrix's first solve). The
 * results are the same bit for bit either way; off runs every sweep as its own launch. Process-wide,
 * like b2g_set_profiling. No counterpart in the reference. */
B2G_API b2g_status b2g_set_sweep_pipeline(int on);
/* The part rule of the multi-part Gauss-Seidel sweep for meshes created after the call: one part (a
 * persistent CTA walking a contiguous cell range) per `cells` cells of a level's average depth, at
 * most one per SM (48 by default, measured best for one solve on the GPU; a batch, whose cases fill
 * the GPU together, wants fewer parts). Results are the same bit for bit for every rule. 1 <= cells
 * <= 65536; process-wide. No counterpart in the reference. */
B2G_API b2g_status b2g_set_part_cells(int cells);

/* Diagnostic: one Gauss-Seidel sweep of `level` (device pointers) recording into the device array
 * `trace` [8 * nChunks + 4 * nParts + 2 * nParts * (maxDepth + 2)] (SM-cycle stamps): per schedule
 * chunk four of the first compute thread (chunk start, past the depth barrier, data ready, row
 * computed); per part {globaltimer ns, SM cycles} at its start and end; per chunk four of the
 * staging warps (bulk copies started, issued, gathers past their waits, gathers issued); per part
 * and depth d two (d published to the downstream parts, upstream parts first seen at d).
 * `schedule` (host, may be NULL) receives {nParts, nChunks, chunk cell capacity, chunk entry
 * capacity, max depth}. */
/* Diagnostic, for testing that the sweep's device-side waits end: one Gauss-Seidel sweep of `level`
 * (device pointers) in which no part publishes its progress, every wait limited to `spinLimit` polls
 * (1 .. 2^24). A part that needs values of another part waits for a progress word nothing sets,
 * gives up, and the call returns B2G_ERR_DEVICE_TIMEOUT with psi invalid; the context stays usable.
 * A level swept by one part has no such wait and returns B2G_OK. *nParts (may be NULL) receives the
 * level's part count. No counterpart in the reference. */
B2G_API b2g_status b2g_level_smooth_stall(b2g_matrix* m, int level, double* psi, const double* source,
                                          long long spinLimit, int* nParts);
/* The grid form of the pipelined sweeps (ranks above 16 CTAs, nSweeps at least 2) with no rank
 * publishing its progress: every wait for a neighbour rank runs out after spinLimit polls, the kernel
 * ends, and the call returns B2G_ERR_DEVICE_TIMEOUT with the context still usable. psi is left in an
 * unspecified state. For tests of the waits' limit. */
B2G_API b2g_status b2g_level_grid_stall(b2g_matrix* m, int level, double* psi, const double* source, int nSweeps,
                                        int ranks, long long spinLimit);
/* nSweeps exact Gauss-Seidel sweeps of `level` (device pointers, natural cell order) in ONE
 * pipelined launch on `ranks` CTAs holding psi in shared memory (1, 2, 4, 8 or 16; a thread-block
 * cluster when above 1), on `ranks` CTAs of the grid form when above 16 (psi in global memory, every
 * CTA resident, each waiting for its neighbour ranks only), or with ranks = -1 as the level's
 * multi-part sweep over (sweep, cell) items, whatever form the level's tuned choice would take: sweep
 * s+1 runs on a cell once every value its row reads is final, which gives bit for bit the result of
 * nSweeps sequential sweeps (gaussSeidelSweeps, smooth_solver_cpp.cu:87-166, called nSweeps times).
 * B2G_ERR_ARGUMENT when the level's cells do not fit that many CTAs' shared memory, such a cluster or
 * grid cannot be resident, or (ranks -1) the level has one part or nSweeps is 1; B2G_ERR_DEVICE_TIMEOUT
 * when a grid-form wait gave up. For tests and tuning. */
B2G_API b2g_status b2g_level_smooth_pipelined(b2g_matrix* m, int level, double* psi, const double* source,
                                              int nSweeps, int ranks);
/* psi = A^-1 source on the coarsest level by its dense Cholesky factor (device pointers, natural
 * cell order): the direct coarsest solve the FP32-preconditioned forms take (coarsestDirect).
 * B2G_ERR_ARGUMENT when the level has more than 96 cells or is not positive definite. The factor of
 * the matrix's current coefficients is made on first use. For tests. */
B2G_API b2g_status b2g_coarsest_dense_solve(b2g_matrix* m, double* psi, const double* source);
/* The tuned choice for smoothing calls of nSweeps sweeps on `level` in values of `valueBytes` (8 FP64,
 * 4 FP32): *ranks the pipelined launch's CTAs (holding psi in shared memory, or of the grid form when
 * *gridForm is 1), or minus the part count of the pipelined multi-part sweep over (sweep, cell) items
 * (0: sweep by sweep, or not tuned yet), *nSteps its combined steps, and the measured milliseconds
 * per call of the chosen pipelined form (else the best shared-memory shape), of the sweep-by-sweep
 * launches, of the best shared-memory shape, of the item schedule and of the best grid form (0: not
 * tried). Any output may be NULL. */
B2G_API b2g_status b2g_level_pipe_shape(const b2g_mesh* mesh, int level, int nSweeps, int valueBytes, int* ranks,
                                        int* nSteps, float* msPipe, float* msSweeps, float* msShared,
                                        float* msItems, float* msGrid, int* gridForm);
B2G_API b2g_status b2g_level_smooth_trace(b2g_matrix* m, int level, double* psi, const double* source,
                                          unsigned long long* trace, int traceCapacity, int* schedule);
/* Diagnostic: the Gauss-Seidel schedule of `level` to HOST arrays (either may be NULL):
 * partChunkStart [nParts + 1] and the chunk records [12 * nChunks] (positions, sweep entries,
 * gathers, depth, upstream depth, same-part wait, depth change, blob offsets). */
B2G_API b2g_status b2g_level_schedule(const b2g_mesh* mesh, int level, int* partChunkStart, int* chunkRecords);

/* ---- the step before the solve ------------------------------------------------------------------ */

/* foldBoundary (gamg_solver_cpp.cu:769-797, fvMatrix::solveSegregated's addBoundaryDiag and
 * addBoundarySource) on the device: the nBFaces boundary faces of all patches concatenated in patch
 * order, each with its cell (faceCells), internal and boundary coefficient and a flag that is
 * nonzero where its patch is coupled. diag [nCells] (the matrix's) becomes the folded diagonal:
 * plus every face's internal coefficient; source [nCells] plus the uncoupled faces' boundary
 * coefficients, added per cell in (patch, face) order as the reference's loop does. All arrays in
 * `memspace`; diag and source in/out. */
B2G_API b2g_status b2g_fold_boundary(int nCells, int nBFaces, const int32_t* faceCells, const double* internalCoeffs,
                                     const double* boundaryCoeffs, const unsigned char* coupled, double* diag,
                                     double* source, int memspace, void* stream);

/* The pressure equation ahead of the solve, on the device: simpleFoam's pEqn.H stages 4-5 as the
 * reference's cpu::assemblePEqn computes them (src/applications/solvers/simpleFoam/pEqn_cpp.cu:209-260)
 * on an orthogonal mesh with uncoupled patches -- fvm::laplacian(fvc::interpolate(rAU), p) ==
 * fvc::div(phiHbyA), then setReference -- bit for bit. The mesh gives the internal faces' addressing;
 * per internal face the linear-interpolation weights, deltaCoeffs, |Sf| and phiHbyA, per cell V and
 * rAU; the boundary faces patch by patch with their cell, |Sf|, deltaCoeffs, pressure condition
 * (bType 1 fixedValue bValue, 0 zeroGradient, 2 empty: left out of the divergence) and phiHbyA;
 * pRefCell -1 for no reference. Out: diag, upper (== lower) and source, and per boundary face the
 * internalCoeffs and boundaryCoeffs that b2g_fold_boundary folds in before the solve. All arrays in
 * `memspace`. A non-orthogonal correction and coupled patches are not assembled here. */
B2G_API b2g_status b2g_assemble_pressure(b2g_mesh* mesh, const double* weights, const double* deltaCoeffs,
                                         const double* magSf, const double* V, const double* rAU,
                                         const double* phiHbyA, int nBFaces, const int32_t* bFaceCells,
                                         const double* bMagSf, const double* bDeltaCoeffs, const int32_t* bType,
                                         const double* bValue, const double* bPhiHbyA, int pRefCell,
                                         double pRefValue, double* diag, double* upper, double* source,
                                         double* internalCoeffs, double* boundaryCoeffs, int memspace,
                                         void* stream);

/* ---- the batched form: many independent cases in one solve ------------------------------------ */

/* A batch of matrices (each on its own mesh), solved together: every step of every level is one
 * launch over all the cases that have that level (levels aligned from the finest), the coarsest
 * solves run one warp per case in one launch, and each PCG iteration is one CUDA graph. Each case's
 * result is the one b2g_matrix_pcg_solve gives: bit for bit with serial-order reductions; with tree
 * reductions the sums are shaped per 2048-cell tile (the same alone or in any batch). No counterpart
 * in the reference's solver interface. The matrices must outlive the batch; the batch runs on a
 * stream of its own. */
typedef struct b2g_batch b2g_batch;
B2G_API b2g_status b2g_batch_create(b2g_matrix* const* matrices, int count, b2g_batch** out);
/* Solves every case (controls->solver must be PCG + GAMG; both precision forms): sources[k] and
 * psis[k] are case k's fields in natural cell order in `memspace`, psis[k] overwritten with the
 * solution; perfs[count] receives each case's SolverPerformance. */
B2G_API b2g_status b2g_batch_solve(b2g_batch* batch, const double* const* sources, double* const* psis,
                                   const b2g_controls* controls, int memspace, b2g_perf* perfs);
/* Kernel launches of the last b2g_batch_solve (a graph replay counts its launches). */
B2G_API b2g_status b2g_batch_launches(const b2g_batch* batch, long long* launches);
B2G_API b2g_status b2g_batch_destroy(b2g_batch* batch);

/* ---- the serving form: many independent cases, solves queued as they arrive ------------------ */

/* A request loop on the current device (no counterpart in the reference's solver interface; it
 * serves the PCG + GAMG solve to many cases at once). nSlots worker threads, each with its own
 * stream and a size class it serves first (slot i: class i mod 3; classes below 2^18 cells, below
 * 2^22, larger), take the oldest queued request of that class (else of any class) together with the
 * queued requests of other idle cases of its class (at most 64, 16 and 4 cases) and controls,
 * and solve the group as one batch (b2g_batch_*: each level step one launch over all of them, each
 * PCG iteration one CUDA graph). Requests that arrive while others are on the GPU join the next
 * group, and the slots' groups overlap on the device. A case is solved by one slot at a time; its
 * result is the same in any group (b2g_batch_solve's). Standalone GAMG requests and requests with a
 * smoother other than GaussSeidel are solved alone (the single-case solve). */
typedef struct b2g_server b2g_server;
B2G_API b2g_status b2g_server_create(unsigned long long hbmCapBytes, int nSlots, b2g_server** out);
/* Stops the workers (queued requests are dropped) and frees every case. */
B2G_API b2g_status b2g_server_destroy(b2g_server* server);
/* Registers a case: builds its hierarchy and its matrix (FP64 and FP32 levels) and keeps both
 * resident, admitted by their HBM footprint: idle cases without queued requests are evicted, least
 * recently used first, until the case fits under the cap; else B2G_ERR_NO_MEMORY. Arguments as
 * b2g_mesh_create and b2g_matrix_create (folded diagonal, upper == lower coefficients). */
B2G_API b2g_status b2g_server_add_case(b2g_server* server, int nCells, int nFaces, const int32_t* lower,
                                       const int32_t* upper, const double* Sf, const double* magSf,
                                       const double* diag, const double* upperCoef, int nCellsInCoarsestLevel,
                                       int memspace, int* caseId);
/* Queues one solve of case `caseId`. `source` (HOST, [nCells]) is read and `psi` (HOST, [nCells])
 * holds the initial guess on entry and the solution once b2g_server_wait has returned for the ticket.
 * Both are the caller's buffers, used in place: they must stay valid, and psi untouched, until then.
 * controls->solver picks PCG + GAMG or GAMG. */
B2G_API b2g_status b2g_server_submit(b2g_server* server, int caseId, const double* source, double* psi,
                                     const b2g_controls* controls, long long* ticket);
/* Waits for a request (timeoutMs < 0: as long as it takes): `out` receives the SolverPerformance,
 * latencyMs the time from submit to result. Returns the solve's own status; B2G_ERR_STATE with
 * "still pending" if the request has not finished at the timeout (its buffers stay in use). */
B2G_API b2g_status b2g_server_wait(b2g_server* server, long long ticket, b2g_perf* out, double* latencyMs,
                                   int timeoutMs);
/* The HBM footprint a case was admitted with (bytes). */
B2G_API b2g_status b2g_server_case_bytes(b2g_server* server, int caseId, unsigned long long* bytes);

/* Diagnostic: the multicolour layout of `level` (B2G_PRECISION_FP32_PRECOND_MULTICOLOUR; built on
 * that form's first solve on the mesh): *nColours (0 if not built yet) and, if colourStart is not
 * NULL, the colours' row ranges colourStart[nColours + 1] (HOST; rows padded to 32 per colour). */
B2G_API b2g_status b2g_level_colouring(const b2g_mesh* mesh, int level, int* nColours, int* colourStart);

/* Diagnostic: the launch shape the autotuner chose for `level`'s multicolour sweep (measured on the
 * form's first solve on the mesh): *wholeLevelCtas 1 if one block sweeps the whole level, c > 1 if
 * one thread-block cluster of c CTAs does, 0 for one launch per colour; *threadsPerBlock the CTAs'
 * size; *msPerSweep the measured time of one sweep. All 0 before. */
B2G_API b2g_status b2g_level_sweep_shape(const b2g_mesh* mesh, int level, int* wholeLevelCtas,
                                         int* threadsPerBlock, float* msPerSweep);
/* Diagnostic: for `level`'s multicolour smoothing calls of nSweeps sweeps (symmetric 1 for
 * symGaussSeidel), whether they run as one pipelined launch whose steps are the colours: *ranks its
 * CTAs (one, or a thread-block cluster), 0 if the colour-by-colour shape above was faster or the
 * level is not pipelined; *msPipe the best pipelined shape's measured time per call (0: not tried);
 * *msColours the colour-by-colour shape's. All 0 before the form's first solve. Any output may be
 * NULL. */
B2G_API b2g_status b2g_level_mc_pipe(const b2g_mesh* mesh, int level, int nSweeps, int symmetric, int* ranks,
                                     float* msPipe, float* msColours);

/* Library version string. */
B2G_API const char* b2g_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BRAE_GAMG_H */
