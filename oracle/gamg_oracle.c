/*
 * gamg_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product). A plain-C
 * restatement of the reference's host GAMG-PCG path; see gamg_oracle.h for the citation keys
 * (AGG, GAMG, SMO) and for how it is pinned. Every floating-point expression keeps the
 * reference's operand order and association, because the hierarchy's integer decisions and the
 * iteration counts depend on the last bit.
 */
#include "gamg_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define SMALL 1e-20   /* solverPerformance::small_ (GAMG:16) */
#define VSMALL 1e-300 /* solverPerformance::vsmall_ (GAMG:17) */
#define GREAT_PERF 1e+20 /* SolverPerformance great_ (GAMG:19) */
#define GREAT_AGG 1.0e+15 /* scalar.H GREAT (AGG:15) */
#define MAX_LEVELS 50 /* GAMGAgglomeration.C:248 (AGG:13) */

enum { SM_GS = 0, SM_SYMGS = 1, SM_DIC = 2, SM_DICGS = 3 };

static void* xmalloc(size_t n)
{
    void* p = malloc(n ? n : 1);
    if (!p)
    {
        fprintf(stderr, "gamg_oracle: out of memory (%zu bytes)\n", n);
        abort();
    }
    return p;
}
static void* xcalloc(size_t n, size_t s)
{
    void* p = calloc(n ? n : 1, s);
    if (!p)
    {
        fprintf(stderr, "gamg_oracle: out of memory\n");
        abort();
    }
    return p;
}

/* ------------------------------------------------------------------------------------------------
 * Agglomeration
 * ----------------------------------------------------------------------------------------------*/

typedef struct
{
    int nCells;
    int nFaces;
    int* lower;
    int* upper;
} oc_addr;

struct oc_agglom
{
    oc_addr fine;
    int nLevels;
    oc_addr levels[MAX_LEVELS];        /* addressing of level i+1 */
    int* restrictAddr[MAX_LEVELS];     /* step i: nCells of level i */
    int* faceRestrict[MAX_LEVELS];     /* step i: nFaces of level i */
    char* flip[MAX_LEVELS];
    double* weights[MAX_LEVELS];       /* weights compared by step i's pairing */
};

static const oc_addr* mesh_level(const oc_agglom* a, int i)
{
    return i == 0 ? &a->fine : &a->levels[i - 1];
}

/* gamgPairAgglomerate (AGG:158-284): one greedy pairing pass; flips *forward on the way out. */
static int* pair_agglomerate(int* nCoarseOut, const oc_addr* fine, const double* w, int* forward)
{
    const int n = fine->nCells;
    const int nF = fine->nFaces;
    const int* up = fine->upper;
    const int* lo = fine->lower;
    /* cellFaces: faces where the cell is UPPER first, then those it owns, each in face order
       (AGG:166-201) */
    int* off = (int*)xcalloc((size_t)n + 1, sizeof(int));
    int* cnt = (int*)xcalloc((size_t)n, sizeof(int));
    int* cf = (int*)xmalloc(sizeof(int) * (size_t)(2 * (size_t)nF));
    for (int f = 0; f < nF; ++f) ++cnt[up[f]];
    for (int f = 0; f < nF; ++f) ++cnt[lo[f]];
    for (int c = 0; c < n; ++c) off[c + 1] = off[c] + cnt[c];
    memset(cnt, 0, sizeof(int) * (size_t)n);
    for (int f = 0; f < nF; ++f) { const int c = up[f]; cf[off[c] + cnt[c]++] = f; }
    for (int f = 0; f < nF; ++f) { const int c = lo[f]; cf[off[c] + cnt[c]++] = f; }

    int* map = (int*)xmalloc(sizeof(int) * (size_t)n);
    for (int c = 0; c < n; ++c) map[c] = -1;
    int nCoarse = 0;
    for (int cfi = 0; cfi < n; ++cfi)
    {
        const int c = *forward ? cfi : n - cfi - 1;
        if (map[c] >= 0) continue;
        int match = -1;
        double maxW = -GREAT_AGG;
        for (int k = off[c]; k < off[c + 1]; ++k)
        {
            const int f = cf[k];
            if (map[up[f]] < 0 && map[lo[f]] < 0 && w[f] > maxW)
            {
                match = f;
                maxW = w[f];
            }
        }
        if (match >= 0)
        {
            map[up[match]] = nCoarse;
            map[lo[match]] = nCoarse;
            ++nCoarse;
            continue;
        }
        /* no unmatched neighbour: join the cluster across the heaviest face (AGG:239-257) */
        int cmatch = -1;
        double cmax = -GREAT_AGG;
        for (int k = off[c]; k < off[c + 1]; ++k)
        {
            const int f = cf[k];
            if (w[f] > cmax)
            {
                cmatch = f;
                cmax = w[f];
            }
        }
        if (cmatch >= 0)
        {
            const int a = map[up[cmatch]];
            const int b = map[lo[cmatch]];
            map[c] = a > b ? a : b;
        }
    }
    /* leftovers become singletons, in visit order (AGG:260-269) */
    for (int cfi = 0; cfi < n; ++cfi)
    {
        const int c = *forward ? cfi : n - cfi - 1;
        if (map[c] < 0) map[c] = nCoarse++;
    }
    if (!*forward)
    {
        /* backward passes renumber c -> nCoarse-1-c (AGG:271-279) */
        --nCoarse;
        for (int c = 0; c < n; ++c) map[c] = nCoarse - map[c];
        ++nCoarse;
    }
    *forward = !*forward;
    free(off);
    free(cnt);
    free(cf);
    *nCoarseOut = nCoarse;
    return map;
}

/* agglomerateLduAddressing (AGG:28-154): coarse faces numbered owner-major, each owner's faces in
 * the order the fine-face walk first met them; face restrict and flip maps. */
static int agglomerate_ldu(oc_agglom* a, int li, int nCoarse)
{
    const oc_addr* fm = mesh_level(a, li);
    const int nFF = fm->nFaces;
    const int* up = fm->upper;
    const int* lo = fm->lower;
    const int* rm = a->restrictAddr[li];

    int* head = (int*)xmalloc(sizeof(int) * (size_t)nCoarse);
    int* tail = (int*)xmalloc(sizeof(int) * (size_t)nCoarse);
    int* cnt = (int*)xcalloc((size_t)nCoarse, sizeof(int));
    for (int c = 0; c < nCoarse; ++c) head[c] = tail[c] = -1;
    int* next = (int*)xmalloc(sizeof(int) * (size_t)(nFF ? nFF : 1));
    int* initNei = (int*)xmalloc(sizeof(int) * (size_t)(nFF ? nFF : 1));
    int* fr = (int*)xmalloc(sizeof(int) * (size_t)(nFF ? nFF : 1));
    int nCF = 0;
    for (int f = 0; f < nFF; ++f)
    {
        const int ru = rm[up[f]];
        const int rl = rm[lo[f]];
        if (ru == rl)
        {
            fr[f] = -(ru + 1);
            continue;
        }
        const int own = ru < rl ? ru : rl;
        const int nei = ru < rl ? rl : ru;
        int found = -1;
        for (int k = head[own]; k >= 0; k = next[k])
        {
            if (initNei[k] == nei)
            {
                found = k;
                break;
            }
        }
        if (found >= 0)
        {
            fr[f] = found;
            continue;
        }
        initNei[nCF] = nei;
        next[nCF] = -1;
        if (tail[own] >= 0) next[tail[own]] = nCF; else head[own] = nCF;
        tail[own] = nCF;
        ++cnt[own];
        fr[f] = nCF;
        ++nCF;
    }
    oc_addr* co = &a->levels[li];
    co->nCells = nCoarse;
    co->nFaces = nCF;
    co->lower = (int*)xmalloc(sizeof(int) * (size_t)(nCF ? nCF : 1));
    co->upper = (int*)xmalloc(sizeof(int) * (size_t)(nCF ? nCF : 1));
    int* cmap = (int*)xmalloc(sizeof(int) * (size_t)(nCF ? nCF : 1));
    int cfi = 0;
    for (int c = 0; c < nCoarse; ++c)
    {
        for (int k = head[c]; k >= 0; k = next[k])
        {
            co->lower[cfi] = c;
            co->upper[cfi] = initNei[k];
            cmap[k] = cfi;
            ++cfi;
        }
    }
    for (int f = 0; f < nFF; ++f)
    {
        if (fr[f] >= 0) fr[f] = cmap[fr[f]];
    }
    char* flip = (char*)xcalloc((size_t)(nFF ? nFF : 1), 1);
    for (int f = 0; f < nFF; ++f)
    {
        const int cfc = fr[f];
        if (cfc < 0) continue;
        const int own = co->lower[cfc];
        const int nei = co->upper[cfc];
        const int ru = rm[up[f]];
        const int rl = rm[lo[f]];
        if (own == ru && nei == rl) flip[f] = 1;
        else if (!(own == rl && nei == ru))
        {
            fprintf(stderr, "gamg_oracle: inconsistent face restriction at face %d level %d\n", f, li);
            abort();
        }
    }
    a->faceRestrict[li] = fr;
    a->flip[li] = flip;
    free(head);
    free(tail);
    free(cnt);
    free(next);
    free(initNei);
    free(cmap);
    return nCF;
}

static int* copy_ints(const int* s, int n)
{
    int* d = (int*)xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    if (n) memcpy(d, s, sizeof(int) * (size_t)n);
    return d;
}

/* faceAreaPairGamgAgglomeration (AGG:286-345) */
oc_agglom* oc_agglomerate(int nCells, int nFaces, const int* lower, const int* upper,
                          const double* Sf, const double* magSf, int nCellsInCoarsestLevel,
                          int* forward)
{
    oc_agglom* a = (oc_agglom*)xcalloc(1, sizeof(oc_agglom));
    a->fine.nCells = nCells;
    a->fine.nFaces = nFaces;
    a->fine.lower = copy_ints(lower, nFaces);
    a->fine.upper = copy_ints(upper, nFaces);

    /* GAMGAgglomeration.C:285 (AGG:297) */
    int half = nCells / 2;
    int nCoarsest = nCellsInCoarsestLevel < half ? nCellsInCoarsestLevel : half;
    if (nCoarsest < 1) nCoarsest = 1;

    /* mag(cmptMultiply(Sf/sqrt(magSf), (1, 1.01, 1.02))) (AGG:301-311) */
    double* w = (double*)xmalloc(sizeof(double) * (size_t)(nFaces ? nFaces : 1));
    for (int f = 0; f < nFaces; ++f)
    {
        const double r = sqrt(magSf[f]);
        const double wx = Sf[3 * (size_t)f] / r;
        const double wy = (Sf[3 * (size_t)f + 1] / r) * 1.01;
        const double wz = (Sf[3 * (size_t)f + 2] / r) * 1.02;
        w[f] = sqrt(wx * wx + wy * wy + wz * wz);
    }

    int nCreated = 0;
    while (nCreated < MAX_LEVELS - 1)
    {
        const oc_addr* fm = mesh_level(a, nCreated);
        int nCoarse = -1;
        int* map = pair_agglomerate(&nCoarse, fm, w, forward);
        /* continueAgglomerating (AGG:17-24) */
        if (nCoarse < nCoarsest || !(nCoarse < fm->nCells))
        {
            free(map);
            break;
        }
        a->restrictAddr[nCreated] = map;
        a->weights[nCreated] = w;
        const int nCF = agglomerate_ldu(a, nCreated, nCoarse);
        /* restrictFaceField: sums over the merged faces in ascending fine face (AGG:328-339) */
        double* cw = (double*)xcalloc((size_t)(nCF ? nCF : 1), sizeof(double));
        const int* fr = a->faceRestrict[nCreated];
        for (int f = 0; f < fm->nFaces; ++f)
        {
            if (fr[f] >= 0) cw[fr[f]] += w[f];
        }
        w = cw;
        ++nCreated;
    }
    free(w);
    a->nLevels = nCreated;
    return a;
}

void oc_agglom_free(oc_agglom* a)
{
    if (!a) return;
    free(a->fine.lower);
    free(a->fine.upper);
    for (int i = 0; i < a->nLevels; ++i)
    {
        free(a->levels[i].lower);
        free(a->levels[i].upper);
        free(a->restrictAddr[i]);
        free(a->faceRestrict[i]);
        free(a->flip[i]);
        free(a->weights[i]);
    }
    free(a);
}

int oc_agglom_nlevels(const oc_agglom* a) { return a->nLevels; }

void oc_agglom_level_size(const oc_agglom* a, int level, int* nCells, int* nFaces)
{
    const oc_addr* m = mesh_level(a, level);
    *nCells = m->nCells;
    *nFaces = m->nFaces;
}

void oc_agglom_get(const oc_agglom* a, int step, int* restrictAddr, int* faceRestrict, char* flip,
                   int* coarseLower, int* coarseUpper)
{
    const oc_addr* fm = mesh_level(a, step);
    const oc_addr* cm = &a->levels[step];
    if (restrictAddr) memcpy(restrictAddr, a->restrictAddr[step], sizeof(int) * (size_t)fm->nCells);
    if (faceRestrict) memcpy(faceRestrict, a->faceRestrict[step], sizeof(int) * (size_t)fm->nFaces);
    if (flip) memcpy(flip, a->flip[step], (size_t)fm->nFaces);
    if (coarseLower) memcpy(coarseLower, cm->lower, sizeof(int) * (size_t)cm->nFaces);
    if (coarseUpper) memcpy(coarseUpper, cm->upper, sizeof(int) * (size_t)cm->nFaces);
}

void oc_agglom_weights(const oc_agglom* a, int step, double* w)
{
    const oc_addr* fm = mesh_level(a, step);
    memcpy(w, a->weights[step], sizeof(double) * (size_t)fm->nFaces);
}

/* ------------------------------------------------------------------------------------------------
 * One LDU level
 * ----------------------------------------------------------------------------------------------*/

typedef struct
{
    int nCells;
    int nFaces;
    const int* lower;
    const int* upper;
    double* diag;
    double* coef; /* upper == lower (symmetric) */
    /* the coupled (cyclic) pair, each face once from its own side (LduLevel::ifOwn/ifNbr/ifCoeff,
     * GAMG:25-36), in the sign convention Amul subtracts; nIf 0 = none */
    int nIf;
    const int* ifOwn;
    const int* ifNbr;
    const double* ifCoeff;
} oc_level;

/* lduMatrix::Amul (GAMG:62-88) */
static void amul_l(const oc_level* A, const double* psi, double* Apsi)
{
    for (int c = 0; c < A->nCells; ++c) Apsi[c] = A->diag[c] * psi[c];
    for (int f = 0; f < A->nFaces; ++f)
    {
        const int u = A->upper[f];
        const int l = A->lower[f];
        Apsi[u] += A->coef[f] * psi[l];
        Apsi[l] += A->coef[f] * psi[u];
    }
    /* the pair, as updateMatrixInterfaces applies it (GAMG:82-87) */
    for (int f = 0; f < A->nIf; ++f) Apsi[A->ifOwn[f]] -= A->ifCoeff[f] * psi[A->ifNbr[f]];
}

/* lduMatrix::residual (GAMG:90-117); rA may alias source */
static void residual_l(const oc_level* A, double* rA, const double* psi, const double* source)
{
    for (int c = 0; c < A->nCells; ++c) rA[c] = source[c] - A->diag[c] * psi[c];
    for (int f = 0; f < A->nFaces; ++f)
    {
        const int u = A->upper[f];
        const int l = A->lower[f];
        rA[u] -= A->coef[f] * psi[l];
        rA[l] -= A->coef[f] * psi[u];
    }
    /* the pair, with the sign Amul's term does not have (GAMG:110-115) */
    for (int f = 0; f < A->nIf; ++f) rA[A->ifOwn[f]] += A->ifCoeff[f] * psi[A->ifNbr[f]];
}

/* lduMatrix::solver::normFactor (GAMG:119-159) */
static double norm_factor_l(const oc_level* A, const double* psi, const double* source,
                            const double* Apsi, double* tmp)
{
    for (int c = 0; c < A->nCells; ++c) tmp[c] = A->diag[c];
    for (int f = 0; f < A->nFaces; ++f)
    {
        tmp[A->upper[f]] += A->coef[f];
        tmp[A->lower[f]] += A->coef[f];
    }
    /* sumA takes the pair with Amul's sign (GAMG:137-145) */
    for (int f = 0; f < A->nIf; ++f) tmp[A->ifOwn[f]] -= A->ifCoeff[f];
    double average = 0;
    for (int c = 0; c < A->nCells; ++c) average += psi[c];
    average /= (double)A->nCells;
    double sum = 0;
    for (int c = 0; c < A->nCells; ++c)
    {
        const double t = tmp[c] * average;
        sum += fabs(Apsi[c] - t) + fabs(source[c] - t);
    }
    return sum + SMALL;
}

/* sumMag, sumProd (GAMG:161-181) */
double oc_sum_mag(int n, const double* x)
{
    double s = 0;
    for (int i = 0; i < n; ++i) s += fabs(x[i]);
    return s;
}
double oc_sum_prod(int n, const double* a, const double* b)
{
    double s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* SolverPerformance::checkConvergence (GAMG:183-191) */
static int converged(const oc_perf* p, double tol, double relTol)
{
    return p->finalResidual < tol || (relTol > SMALL && p->finalResidual < relTol * p->initialResidual);
}

/* DICPreconditioner::calcReciprocalD (GAMG:194-210) */
static double* dic_rD(const oc_level* A)
{
    double* rD = (double*)xmalloc(sizeof(double) * (size_t)A->nCells);
    memcpy(rD, A->diag, sizeof(double) * (size_t)A->nCells);
    for (int f = 0; f < A->nFaces; ++f)
    {
        rD[A->upper[f]] -= A->coef[f] * A->coef[f] / rD[A->lower[f]];
    }
    for (int c = 0; c < A->nCells; ++c) rD[c] = 1.0 / rD[c];
    return rD;
}

/* the DIC substitution passes on w = rD*r (GAMG:212-231) */
static void dic_substitute(const oc_level* A, const double* rD, double* w)
{
    for (int f = 0; f < A->nFaces; ++f)
    {
        const int u = A->upper[f];
        w[u] -= rD[u] * A->coef[f] * w[A->lower[f]];
    }
    for (int f = A->nFaces; f-- > 0;)
    {
        const int l = A->lower[f];
        w[l] -= rD[l] * A->coef[f] * w[A->upper[f]];
    }
}

/* lduOwnerStart (SMO:10-34) */
static int* owner_start(const oc_level* A)
{
    int* os = (int*)xcalloc((size_t)A->nCells + 1, sizeof(int));
    for (int f = 0; f < A->nFaces; ++f)
    {
        if (A->lower[f] >= A->upper[f] || (f > 0 && A->lower[f] < A->lower[f - 1]))
        {
            fprintf(stderr, "gamg_oracle: face %d breaks upper-triangular order\n", f);
            abort();
        }
        ++os[A->lower[f] + 1];
    }
    for (int c = 0; c < A->nCells; ++c) os[c + 1] += os[c];
    return os;
}

/* gaussSeidelSweeps without interfaces (SMO:87-166): the ascending walk gathers upper*psi over
 * owned faces and distributes lower*psi into bPrime; the symmetric variant adds a descending walk
 * that reuses bPrime and does not distribute. */
static void gs_sweeps(const oc_level* A, const int* os, const double* b, double* psi, int nSweeps,
                      int symmetric, double* bPrime)
{
    const int n = A->nCells;
    const int* nei = A->upper;
    for (int s = 0; s < nSweeps; ++s)
    {
        memcpy(bPrime, b, sizeof(double) * (size_t)n);
        for (int c = 0; c < n; ++c)
        {
            const int fs = os[c];
            const int fe = os[c + 1];
            double psii = bPrime[c];
            for (int f = fs; f < fe; ++f) psii -= A->coef[f] * psi[nei[f]];
            psii /= A->diag[c];
            for (int f = fs; f < fe; ++f) bPrime[nei[f]] -= A->coef[f] * psii;
            psi[c] = psii;
        }
        if (!symmetric) continue;
        for (int c = n - 1; c >= 0; --c)
        {
            const int fs = os[c];
            const int fe = os[c + 1];
            double psii = bPrime[c];
            for (int f = fs; f < fe; ++f) psii -= A->coef[f] * psi[nei[f]];
            psii /= A->diag[c];
            psi[c] = psii;
        }
    }
}

/* Smoother::smooth (GAMG:234-317) */
typedef struct
{
    const oc_level* A;
    int kind;
    double* rD;
    int* os;
} oc_smoother;

static void smoother_init(oc_smoother* s, const oc_level* A, int kind)
{
    s->A = A;
    s->kind = kind;
    s->rD = (kind == SM_DIC || kind == SM_DICGS) ? dic_rD(A) : NULL;
    s->os = (kind == SM_GS || kind == SM_SYMGS || kind == SM_DICGS) ? owner_start(A) : NULL;
}
static void smoother_free(oc_smoother* s)
{
    free(s->rD);
    free(s->os);
}
static void smoother_smooth(const oc_smoother* s, double* psi, const double* source, int nSweeps)
{
    const oc_level* A = s->A;
    const int n = A->nCells;
    double* tmp = (double*)xmalloc(sizeof(double) * (size_t)(n ? n : 1));
    if (s->kind == SM_DIC || s->kind == SM_DICGS)
    {
        /* DICSmoother::smooth */
        for (int sw = 0; sw < nSweeps; ++sw)
        {
            residual_l(A, tmp, psi, source);
            for (int i = 0; i < n; ++i) tmp[i] *= s->rD[i];
            dic_substitute(A, s->rD, tmp);
            for (int i = 0; i < n; ++i) psi[i] += tmp[i];
        }
    }
    if (s->kind != SM_DIC)
    {
        /* the pair enters through bPrime, once per smooth() with psi as it stands at entry
         * (GAMG:287-305) */
        double* b = NULL;
        if (A->nIf > 0)
        {
            b = (double*)xmalloc(sizeof(double) * (size_t)(n ? n : 1));
            memcpy(b, source, sizeof(double) * (size_t)n);
            for (int f = 0; f < A->nIf; ++f) b[A->ifOwn[f]] += A->ifCoeff[f] * psi[A->ifNbr[f]];
        }
        gs_sweeps(A, s->os, b ? b : source, psi, nSweeps, s->kind == SM_SYMGS, tmp);
        free(b);
    }
    free(tmp);
}

/* pcgDic (GAMG:321-383): PCG with DIC from the psi handed in; maxIter 1000 on the coarsest level */
static oc_perf pcg_dic_l(const oc_level* A, double* psi, const double* source, double tol,
                         double relTol, int maxIter)
{
    const int n = A->nCells;
    double* pA = (double*)xmalloc(sizeof(double) * (size_t)n);
    double* wA = (double*)xmalloc(sizeof(double) * (size_t)n);
    double* rA = (double*)xmalloc(sizeof(double) * (size_t)n);
    double wArA = GREAT_PERF;
    double wArAold = wArA;
    amul_l(A, psi, wA);
    for (int c = 0; c < n; ++c) rA[c] = source[c] - wA[c];
    const double nf = norm_factor_l(A, psi, source, wA, pA);
    oc_perf perf;
    perf.nIterations = 0;
    perf.initialResidual = oc_sum_mag(n, rA) / nf;
    perf.finalResidual = perf.initialResidual;
    if (!converged(&perf, tol, relTol))
    {
        double* rD = dic_rD(A);
        do
        {
            wArAold = wArA;
            for (int c = 0; c < n; ++c) wA[c] = rD[c] * rA[c];
            dic_substitute(A, rD, wA);
            wArA = oc_sum_prod(n, wA, rA);
            if (perf.nIterations == 0)
            {
                memcpy(pA, wA, sizeof(double) * (size_t)n);
            }
            else
            {
                const double beta = wArA / wArAold;
                for (int c = 0; c < n; ++c) pA[c] = wA[c] + beta * pA[c];
            }
            amul_l(A, pA, wA);
            const double wApA = oc_sum_prod(n, wA, pA);
            if (fabs(wApA) / nf < VSMALL) break;
            const double alpha = wArA / wApA;
            for (int c = 0; c < n; ++c)
            {
                psi[c] += alpha * pA[c];
                rA[c] -= alpha * wA[c];
            }
            perf.finalResidual = oc_sum_mag(n, rA) / nf;
        } while (++perf.nIterations < maxIter && !converged(&perf, tol, relTol));
        free(rD);
    }
    free(pA);
    free(wA);
    free(rA);
    return perf;
}

/* GAMGSolver::scale (GAMG:386-407) */
static void scale_l(const oc_level* A, double* field, double* Acf, const double* source)
{
    amul_l(A, field, Acf);
    double num = 0;
    double den = 0;
    for (int i = 0; i < A->nCells; ++i)
    {
        num += field[i] * source[i];
        den += field[i] * Acf[i];
    }
    const double sf = num / (den >= 0 ? den + VSMALL : den - VSMALL);
    for (int i = 0; i < A->nCells; ++i)
    {
        field[i] = sf * field[i] + (source[i] - sf * Acf[i]) / A->diag[i];
    }
}

/* restrictField / prolongField (GAMG:410-432) */
static void restrict_field(double* cf, int nC, const double* ff, int nF, const int* map)
{
    for (int i = 0; i < nC; ++i) cf[i] = 0;
    for (int i = 0; i < nF; ++i) cf[map[i]] += ff[i];
}
static void prolong_field(double* ff, int nF, const double* cf, const int* map)
{
    for (int i = 0; i < nF; ++i) ff[i] = cf[map[i]];
}

/* ------------------------------------------------------------------------------------------------
 * The hierarchy of matrices: GamgHierarchy::build (GAMG:565-623) with agglomerateMatrix
 * (GAMG:474-526, symmetric branch, no interfaces)
 * ----------------------------------------------------------------------------------------------*/

struct oc_hier
{
    const oc_agglom* a;
    int nLevels;               /* coarse levels */
    oc_level lev[MAX_LEVELS];  /* lev[0] = the folded fine matrix, lev[i] = coarse level i */
};

/* GAMGSolver::agglomerateMatrix's coarse interface (GAMG:497-524): each fine pair face keyed on
 * the coarse cell pair (own, nbr) it joins, in fine face order; a new pair appends a coarse face, a
 * seen one reuses it; the coefficients summed onto it from zero in fine face order. The lookup is an
 * open-addressing table on the pair. */
static void agglomerate_pair(const oc_level* fm, oc_level* cm, const int* restrictAddr)
{
    cm->nIf = 0;
    cm->ifOwn = NULL;
    cm->ifNbr = NULL;
    cm->ifCoeff = NULL;
    if (fm->nIf == 0) return;
    const int nF = fm->nIf;
    int* own = (int*)xmalloc(sizeof(int) * (size_t)nF);
    int* nbr = (int*)xmalloc(sizeof(int) * (size_t)nF);
    double* coeff = (double*)xmalloc(sizeof(double) * (size_t)nF);
    size_t cap = 16;
    while (cap < 2 * (size_t)nF) cap <<= 1;
    int* slot = (int*)xmalloc(sizeof(int) * cap);
    for (size_t i = 0; i < cap; ++i) slot[i] = -1;
    int nC = 0;
    for (int f = 0; f < nF; ++f)
    {
        const int co = restrictAddr[fm->ifOwn[f]];
        const int cn = restrictAddr[fm->ifNbr[f]];
        uint64_t hsh = ((uint64_t)(uint32_t)co * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)(uint32_t)cn * 0xC2B2AE3D27D4EB4Full);
        size_t i = (size_t)(hsh ^ (hsh >> 29)) & (cap - 1);
        while (slot[i] >= 0 && !(own[slot[i]] == co && nbr[slot[i]] == cn)) i = (i + 1) & (cap - 1);
        if (slot[i] < 0)
        {
            slot[i] = nC;
            own[nC] = co;
            nbr[nC] = cn;
            coeff[nC] = 0.0;
            ++nC;
        }
        coeff[slot[i]] += fm->ifCoeff[f];
    }
    free(slot);
    cm->nIf = nC;
    cm->ifOwn = own;
    cm->ifNbr = nbr;
    cm->ifCoeff = coeff;
}

oc_hier* oc_hier_build(const oc_agglom* a, const double* diag, const double* upper)
{
    return oc_hier_build_pair(a, diag, upper, 0, NULL, NULL, NULL);
}

oc_hier* oc_hier_build_pair(const oc_agglom* a, const double* diag, const double* upper, int nIf,
                            const int* ifOwn, const int* ifNbr, const double* ifCoeff)
{
    oc_hier* h = (oc_hier*)xcalloc(1, sizeof(oc_hier));
    h->a = a;
    h->nLevels = a->nLevels;
    oc_level* f0 = &h->lev[0];
    f0->nCells = a->fine.nCells;
    f0->nFaces = a->fine.nFaces;
    f0->lower = a->fine.lower;
    f0->upper = a->fine.upper;
    f0->diag = (double*)xmalloc(sizeof(double) * (size_t)(f0->nCells ? f0->nCells : 1));
    f0->coef = (double*)xmalloc(sizeof(double) * (size_t)(f0->nFaces ? f0->nFaces : 1));
    memcpy(f0->diag, diag, sizeof(double) * (size_t)f0->nCells);
    memcpy(f0->coef, upper, sizeof(double) * (size_t)f0->nFaces);
    f0->nIf = nIf;
    if (nIf > 0)
    {
        int* o = (int*)xmalloc(sizeof(int) * (size_t)nIf);
        int* nb = (int*)xmalloc(sizeof(int) * (size_t)nIf);
        double* cf = (double*)xmalloc(sizeof(double) * (size_t)nIf);
        memcpy(o, ifOwn, sizeof(int) * (size_t)nIf);
        memcpy(nb, ifNbr, sizeof(int) * (size_t)nIf);
        memcpy(cf, ifCoeff, sizeof(double) * (size_t)nIf);
        f0->ifOwn = o;
        f0->ifNbr = nb;
        f0->ifCoeff = cf;
    }
    for (int i = 0; i < a->nLevels; ++i)
    {
        const oc_level* fm = &h->lev[i];
        oc_level* cm = &h->lev[i + 1];
        cm->nCells = a->levels[i].nCells;
        cm->nFaces = a->levels[i].nFaces;
        cm->lower = a->levels[i].lower;
        cm->upper = a->levels[i].upper;
        cm->diag = (double*)xmalloc(sizeof(double) * (size_t)cm->nCells);
        cm->coef = (double*)xcalloc((size_t)(cm->nFaces ? cm->nFaces : 1), sizeof(double));
        restrict_field(cm->diag, cm->nCells, fm->diag, fm->nCells, a->restrictAddr[i]);
        const int* fr = a->faceRestrict[i];
        for (int f = 0; f < fm->nFaces; ++f)
        {
            const int c = fr[f];
            if (c >= 0) cm->coef[c] += fm->coef[f];
            else cm->diag[-1 - c] += 2 * fm->coef[f];
        }
        agglomerate_pair(fm, cm, a->restrictAddr[i]);
    }
    return h;
}

void oc_hier_free(oc_hier* h)
{
    if (!h) return;
    for (int i = 0; i <= h->nLevels; ++i)
    {
        free(h->lev[i].diag);
        free(h->lev[i].coef);
        free((void*)h->lev[i].ifOwn);
        free((void*)h->lev[i].ifNbr);
        free((void*)h->lev[i].ifCoeff);
    }
    free(h);
}

int oc_hier_level_pair(const oc_hier* h, int level, int* ifOwn, int* ifNbr, double* ifCoeff)
{
    const oc_level* L = &h->lev[level];
    if (ifOwn) memcpy(ifOwn, L->ifOwn, sizeof(int) * (size_t)L->nIf);
    if (ifNbr) memcpy(ifNbr, L->ifNbr, sizeof(int) * (size_t)L->nIf);
    if (ifCoeff) memcpy(ifCoeff, L->ifCoeff, sizeof(double) * (size_t)L->nIf);
    return L->nIf;
}

void oc_hier_level(const oc_hier* h, int level, double* diag, double* upper)
{
    const oc_level* L = &h->lev[level];
    memcpy(diag, L->diag, sizeof(double) * (size_t)L->nCells);
    memcpy(upper, L->coef, sizeof(double) * (size_t)L->nFaces);
}

/* ------------------------------------------------------------------------------------------------
 * V-cycle (GAMG:627-735)
 * ----------------------------------------------------------------------------------------------*/

typedef struct
{
    const oc_hier* h;
    oc_smoother sm[MAX_LEVELS + 1]; /* sm[0] finest, sm[i+1] coarse level i+1 */
    double* corr[MAX_LEVELS];       /* coarseCorrFields[i] on coarse level i+1 */
    double* src[MAX_LEVELS];        /* coarseSources[i] */
    double* ACf;
    double* preSmoothed;
} oc_vstate;

static void vstate_init(oc_vstate* v, const oc_hier* h, int smootherKind)
{
    memset(v, 0, sizeof(*v));
    v->h = h;
    int maxN = h->lev[0].nCells;
    for (int i = 0; i <= h->nLevels; ++i) smoother_init(&v->sm[i], &h->lev[i], smootherKind);
    for (int i = 0; i < h->nLevels; ++i)
    {
        const int n = h->lev[i + 1].nCells;
        v->corr[i] = (double*)xcalloc((size_t)n, sizeof(double));
        v->src[i] = (double*)xcalloc((size_t)n, sizeof(double));
    }
    v->ACf = (double*)xcalloc((size_t)maxN, sizeof(double));
    v->preSmoothed = (double*)xcalloc((size_t)maxN, sizeof(double));
}
static void vstate_free(oc_vstate* v)
{
    for (int i = 0; i <= v->h->nLevels; ++i) smoother_free(&v->sm[i]);
    for (int i = 0; i < v->h->nLevels; ++i)
    {
        free(v->corr[i]);
        free(v->src[i]);
    }
    free(v->ACf);
    free(v->preSmoothed);
}

static int imin(int a, int b) { return a < b ? a : b; }

static void vcycle(oc_vstate* v, const oc_controls* c, double* psi, const double* source,
                   double* Apsi, double* finestCorrection, const double* finestResidual,
                   oc_perf* log, int logCap, int* nLog)
{
    const oc_hier* h = v->h;
    const oc_agglom* a = h->a;
    const int coarsest = h->nLevels - 1;
    restrict_field(v->src[0], h->lev[1].nCells, finestResidual, h->lev[0].nCells, a->restrictAddr[0]);
    for (int li = 0; li < coarsest; ++li)
    {
        const oc_level* L = &h->lev[li + 1];
        if (c->nPreSweeps)
        {
            memset(v->corr[li], 0, sizeof(double) * (size_t)L->nCells);
            smoother_smooth(&v->sm[li + 1], v->corr[li], v->src[li],
                            imin(c->nPreSweeps + c->preSweepsLevelMultiplier * li, c->maxPreSweeps));
            if (c->scaleCorrection && li < coarsest - 1) scale_l(L, v->corr[li], v->ACf, v->src[li]);
            residual_l(L, v->src[li], v->corr[li], v->src[li]);
        }
        restrict_field(v->src[li + 1], h->lev[li + 2].nCells, v->src[li], L->nCells,
                       a->restrictAddr[li + 1]);
    }
    {
        const oc_level* L = &h->lev[coarsest + 1];
        memset(v->corr[coarsest], 0, sizeof(double) * (size_t)L->nCells);
        const oc_perf p = pcg_dic_l(L, v->corr[coarsest], v->src[coarsest], c->tolerance, c->relTol, 1000);
        if (log && nLog && *nLog < logCap) log[*nLog] = p;
        if (nLog) ++*nLog;
    }
    for (int li = coarsest - 1; li >= 0; --li)
    {
        const oc_level* L = &h->lev[li + 1];
        if (c->nPreSweeps) memcpy(v->preSmoothed, v->corr[li], sizeof(double) * (size_t)L->nCells);
        prolong_field(v->corr[li], L->nCells, v->corr[li + 1], a->restrictAddr[li + 1]);
        if (c->scaleCorrection && li < coarsest - 1) scale_l(L, v->corr[li], v->ACf, v->src[li]);
        if (c->nPreSweeps)
        {
            for (int i = 0; i < L->nCells; ++i) v->corr[li][i] += v->preSmoothed[i];
        }
        smoother_smooth(&v->sm[li + 1], v->corr[li], v->src[li],
                        imin(c->nPostSweeps + c->postSweepsLevelMultiplier * li, c->maxPostSweeps));
    }
    const oc_level* F = &h->lev[0];
    prolong_field(finestCorrection, F->nCells, v->corr[0], a->restrictAddr[0]);
    if (c->scaleCorrection) scale_l(F, finestCorrection, Apsi, finestResidual);
    for (int i = 0; i < F->nCells; ++i) psi[i] += finestCorrection[i];
    smoother_smooth(&v->sm[0], psi, source, c->nFinestSweeps);
}

/* GAMGPreconditioner::precondition (GAMG:1089-1107) */
static void precondition_v(oc_vstate* v, const oc_controls* c, double* w, const double* r,
                           double* AwA, double* fc, double* fr, oc_perf* log, int cap, int* nLog)
{
    const oc_level* A = &v->h->lev[0];
    const int n = A->nCells;
    memset(w, 0, sizeof(double) * (size_t)n);
    memcpy(fr, r, sizeof(double) * (size_t)n);
    for (int cycle = 0; cycle < c->nVcycles; ++cycle)
    {
        vcycle(v, c, w, r, AwA, fc, fr, log, cap, nLog);
        if (cycle < c->nVcycles - 1)
        {
            amul_l(A, w, AwA);
            for (int i = 0; i < n; ++i)
            {
                fr[i] = r[i];
                fr[i] -= AwA[i];
            }
        }
    }
}

void oc_precondition(const oc_hier* h, const oc_controls* c, double* w, const double* r,
                     oc_perf* coarsest, int cap, int* nCoarsest)
{
    oc_vstate v;
    vstate_init(&v, h, c->smoother);
    const int n = h->lev[0].nCells;
    double* AwA = (double*)xcalloc((size_t)n, sizeof(double));
    double* fc = (double*)xcalloc((size_t)n, sizeof(double));
    double* fr = (double*)xcalloc((size_t)n, sizeof(double));
    if (nCoarsest) *nCoarsest = 0;
    precondition_v(&v, c, w, r, AwA, fc, fr, coarsest, cap, nCoarsest);
    free(AwA);
    free(fc);
    free(fr);
    vstate_free(&v);
}

/* pcgGamgSolveImpl (GAMG:1031-1143), on a folded system */
oc_perf oc_pcg_gamg_solve(const oc_agglom* a, const double* diag, const double* upper,
                          const double* source, double* psi, double tolerance, double relTol,
                          int maxIter, int minIter, const oc_controls* c, double* history,
                          int historyCap, oc_perf* coarsest, int coarsestCap, int* nCoarsest)
{
    const int n = a->fine.nCells;
    oc_level A;
    A.nCells = n;
    A.nFaces = a->fine.nFaces;
    A.lower = a->fine.lower;
    A.upper = a->fine.upper;
    A.diag = (double*)diag;
    A.coef = (double*)upper;
    A.nIf = 0;
    A.ifOwn = NULL;
    A.ifNbr = NULL;
    A.ifCoeff = NULL;
    double* pA = (double*)xcalloc((size_t)n, sizeof(double));
    double* wA = (double*)xcalloc((size_t)n, sizeof(double));
    double* rA = (double*)xcalloc((size_t)n, sizeof(double));
    double wArA = GREAT_PERF;
    double wArAold = wArA;
    if (nCoarsest) *nCoarsest = 0;

    amul_l(&A, psi, wA);
    for (int i = 0; i < n; ++i) rA[i] = source[i] - wA[i];
    const double nf = norm_factor_l(&A, psi, source, wA, pA);
    oc_perf perf;
    perf.nIterations = 0;
    perf.initialResidual = oc_sum_mag(n, rA) / nf;
    perf.finalResidual = perf.initialResidual;
    if (minIter <= 0 && converged(&perf, tolerance, relTol))
    {
        free(pA);
        free(wA);
        free(rA);
        return perf;
    }
    oc_hier* h = oc_hier_build(a, diag, upper);
    oc_vstate v;
    vstate_init(&v, h, c->smoother);
    double* AwA = (double*)xcalloc((size_t)n, sizeof(double));
    double* fc = (double*)xcalloc((size_t)n, sizeof(double));
    double* fr = (double*)xcalloc((size_t)n, sizeof(double));
    do
    {
        wArAold = wArA;
        precondition_v(&v, c, wA, rA, AwA, fc, fr, coarsest, coarsestCap, nCoarsest);
        wArA = oc_sum_prod(n, wA, rA);
        if (perf.nIterations == 0)
        {
            memcpy(pA, wA, sizeof(double) * (size_t)n);
        }
        else
        {
            const double beta = wArA / wArAold;
            for (int i = 0; i < n; ++i) pA[i] = wA[i] + beta * pA[i];
        }
        amul_l(&A, pA, wA);
        const double wApA = oc_sum_prod(n, wA, pA);
        if (fabs(wApA) / nf < VSMALL) break;
        const double alpha = wArA / wApA;
        for (int i = 0; i < n; ++i)
        {
            psi[i] += alpha * pA[i];
            rA[i] -= alpha * wA[i];
        }
        perf.finalResidual = oc_sum_mag(n, rA) / nf;
        if (history && perf.nIterations < historyCap) history[perf.nIterations] = perf.finalResidual;
    } while ((++perf.nIterations < maxIter && !converged(&perf, tolerance, relTol))
             || perf.nIterations < minIter);
    free(AwA);
    free(fc);
    free(fr);
    vstate_free(&v);
    oc_hier_free(h);
    free(pA);
    free(wA);
    free(rA);
    return perf;
}

/* gamgSolveFoldedImpl (GAMG:961-1027) */
oc_perf oc_gamg_solve(const oc_agglom* a, const double* diag, const double* upper,
                      const double* source, double* psi, const oc_controls* c, double* history,
                      int historyCap)
{
    return oc_gamg_solve_pair(a, diag, upper, 0, NULL, NULL, NULL, source, psi, c, history, historyCap);
}

/* gamgSolve (GAMG:943-959) with a coupled pair: gamgLevel0Interface's pair (GAMG:440-470) on the
 * finest level, agglomerated onto every coarse level, on a folded system */
oc_perf oc_gamg_solve_pair(const oc_agglom* a, const double* diag, const double* upper, int nIf,
                           const int* ifOwn, const int* ifNbr, const double* ifCoeff,
                           const double* source, double* psi, const oc_controls* c, double* history,
                           int historyCap)
{
    oc_hier* h = oc_hier_build_pair(a, diag, upper, nIf, ifOwn, ifNbr, ifCoeff);
    const oc_level* F = &h->lev[0];
    const int n = F->nCells;
    double* Apsi = (double*)xcalloc((size_t)n, sizeof(double));
    double* fc = (double*)xcalloc((size_t)n, sizeof(double));
    double* fr = (double*)xcalloc((size_t)n, sizeof(double));
    amul_l(F, psi, Apsi);
    const double nf = norm_factor_l(F, psi, source, Apsi, fc);
    for (int i = 0; i < n; ++i) fr[i] = source[i] - Apsi[i];
    oc_perf perf;
    perf.nIterations = 0;
    perf.initialResidual = oc_sum_mag(n, fr) / nf;
    perf.finalResidual = perf.initialResidual;
    if (!(c->minIter <= 0 && converged(&perf, c->tolerance, c->relTol)))
    {
        oc_vstate v;
        vstate_init(&v, h, c->smoother);
        do
        {
            vcycle(&v, c, psi, source, Apsi, fc, fr, NULL, 0, NULL);
            amul_l(F, psi, Apsi);
            for (int i = 0; i < n; ++i)
            {
                fr[i] = source[i];
                fr[i] -= Apsi[i];
            }
            perf.finalResidual = oc_sum_mag(n, fr) / nf;
            if (history && perf.nIterations < historyCap) history[perf.nIterations] = perf.finalResidual;
        } while ((++perf.nIterations < c->maxIter && !converged(&perf, c->tolerance, c->relTol))
                 || perf.nIterations < c->minIter);
        vstate_free(&v);
    }
    free(Apsi);
    free(fc);
    free(fr);
    oc_hier_free(h);
    return perf;
}

/* ------------------------------------------------------------------------------------------------
 * Flat entry points on one level, for kernel-level parity tests
 * ----------------------------------------------------------------------------------------------*/

static oc_level flat_level(int nC, int nF, const int* lower, const int* upper, const double* diag,
                           const double* coef)
{
    oc_level L;
    L.nCells = nC;
    L.nFaces = nF;
    L.lower = lower;
    L.upper = upper;
    L.diag = (double*)diag;
    L.coef = (double*)coef;
    L.nIf = 0;
    L.ifOwn = NULL;
    L.ifNbr = NULL;
    L.ifCoeff = NULL;
    return L;
}

void oc_amul(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
             const double* coef, const double* psi, double* Apsi)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    amul_l(&L, psi, Apsi);
}

double oc_norm_factor(int nCells, int nFaces, const int* lower, const int* upper,
                      const double* diag, const double* coef, const double* psi,
                      const double* source, const double* Apsi)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    double* tmp = (double*)xmalloc(sizeof(double) * (size_t)(nCells ? nCells : 1));
    const double nf = norm_factor_l(&L, psi, source, Apsi, tmp);
    free(tmp);
    return nf;
}

void oc_smooth(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
               const double* coef, double* psi, const double* source, int nSweeps, int smoother)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    oc_smoother s;
    smoother_init(&s, &L, smoother);
    smoother_smooth(&s, psi, source, nSweeps);
    smoother_free(&s);
}

oc_perf oc_pcg_dic(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
                   const double* coef, double* psi, const double* source, double tolerance,
                   double relTol, int maxIter)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    return pcg_dic_l(&L, psi, source, tolerance, relTol, maxIter);
}

void oc_scale(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
              const double* coef, double* field, double* Acf, const double* source)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    scale_l(&L, field, Acf, source);
}

void oc_amul_pair(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
                  const double* coef, int nIf, const int* ifOwn, const int* ifNbr, const double* ifCoeff,
                  const double* psi, double* Apsi)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    L.nIf = nIf;
    L.ifOwn = ifOwn;
    L.ifNbr = ifNbr;
    L.ifCoeff = ifCoeff;
    amul_l(&L, psi, Apsi);
}

void oc_smooth_pair(int nCells, int nFaces, const int* lower, const int* upper, const double* diag,
                    const double* coef, int nIf, const int* ifOwn, const int* ifNbr, const double* ifCoeff,
                    double* psi, const double* source, int nSweeps, int smoother)
{
    oc_level L = flat_level(nCells, nFaces, lower, upper, diag, coef);
    L.nIf = nIf;
    L.ifOwn = ifOwn;
    L.ifNbr = ifNbr;
    L.ifCoeff = ifCoeff;
    oc_smoother sm;
    smoother_init(&sm, &L, smoother);
    smoother_smooth(&sm, psi, source, nSweeps);
    smoother_free(&sm);
}

/* ------------------------------------------------------------------------------------------------
 * The pressure equation's assembly (cpu::assemblePEqn, pEqn_cpp.cu:209-260), orthogonal, uncoupled
 * ------------------------------------------------------------------------------------------------ */
void oc_assemble_pressure(int nCells, int nFaces, const int* lower, const int* upper, const double* weights,
                          const double* deltaCoeffs, const double* magSf, const double* V, const double* rAU,
                          const double* phi, int nBFaces, const int* bFaceCells, const double* bMagSf,
                          const double* bDeltaCoeffs, const int* bType, const double* bValue,
                          const double* bPhi, int pRefCell, double pRefValue, double* diag, double* coef,
                          double* source, double* internalCoeffs, double* boundaryCoeffs)
{
    int c, f, b;
    double* d = (double*)malloc(sizeof(double) * (size_t)(nCells > 0 ? nCells : 1));
    /* fvm::laplacian(interpolate(rAU), p) (fvm.cuh:130-150, fvc.cu:639-640) */
    for (c = 0; c < nCells; ++c) diag[c] = 0.0;
    for (f = 0; f < nFaces; ++f)
    {
        const double w = weights[f];
        const double rf = w * rAU[lower[f]] + (1.0 - w) * rAU[upper[f]];
        const double k = deltaCoeffs[f] * rf * magSf[f];
        coef[f] = k;
        diag[lower[f]] -= k;
        diag[upper[f]] -= k;
    }
    /* laplacianBoundaryCoeffs (fvm.cuh:40-95): pGamma = rAUf_b*|Sf|, the boundary rAUf being the
     * cell's; fixedValue's gradient coefficients -deltaCoeffs and value*deltaCoeffs, zeroGradient's 0 */
    for (b = 0; b < nBFaces; ++b)
    {
        const double pGamma = rAU[bFaceCells[b]] * bMagSf[b];
        const int fixed = bType[b] == 1;
        const double gIC = fixed ? -bDeltaCoeffs[b] : 0.0;
        const double gBC = fixed ? bValue[b] * bDeltaCoeffs[b] : 0.0;
        internalCoeffs[b] = pGamma * gIC;
        boundaryCoeffs[b] = (-pGamma) * gBC;
    }
    /* the laplacian's own source is zero on an orthogonal mesh; source += div(phiHbyA)*V with
     * div = surfaceIntegrate (fvc.cu:706-730) */
    for (c = 0; c < nCells; ++c) d[c] = 0.0;
    for (f = 0; f < nFaces; ++f)
    {
        d[lower[f]] += phi[f];
        d[upper[f]] -= phi[f];
    }
    for (b = 0; b < nBFaces; ++b)
        if (bType[b] != 2) d[bFaceCells[b]] += bPhi[b];
    for (c = 0; c < nCells; ++c) d[c] /= V[c];
    for (c = 0; c < nCells; ++c) source[c] = 0.0 + d[c] * V[c];
    /* setReference (fvMatrix.C:1011-1023 as pEqn_cpp.cu:248-255 applies it) */
    if (pRefCell >= 0 && pRefCell < nCells)
    {
        source[pRefCell] += diag[pRefCell] * pRefValue;
        diag[pRefCell] += diag[pRefCell];
    }
    free(d);
}
