// batch.cuh -- many independent pressure solves as one: the PCG + GAMG solve of K resident cases
// (each a Matrix on its own mesh hierarchy) with every step of every level one launch over all the
// cases that have that level.
//
// Levels are aligned from the top: mesh level lv of every case runs in the same launches, so the
// sweep counts, which depend on lv alone, agree. A case stops restricting at its own coarsest level;
// the coarsest solves of all cases run in one launch (one warp each) between the way down and the
// way up. Each case keeps its own data where it lies: a launch reads a table of per-case descriptors
// (rows, vectors by role, step maps, scalars) and a tile list, each tile a range of one case's cells.
// Reductions are per case: per tile, then per case over its tiles in a fixed order, so a case's
// results do not depend on which other cases share the batch. The Gauss-Seidel sweep of a level is
// one persistent launch over the concatenated parts of all its cases (gsSweepBatch).
//
// Per-case convergence: each case leaves the iteration as it converges (device-side flags); the
// kernels skip inactive cases, whose fields stay as they were.
#pragma once

#include <map>

#include "solver.cuh"

namespace b2g {

// The vectors of one case on one level, by role (null where the case has none).
enum VecRole : int
{
    V_CORR = 0,  // coarse levels: the correction
    V_SRC,       // coarse levels: the restricted residual
    V_ACF,       // A * field scratch of scale()
    V_PRE,       // pre-smoothed correction scratch
    V_W,         // finest: the preconditioned residual w (the V-cycle's psi)
    V_R,         // finest: the residual r (the V-cycle's source)
    V_AWA,       // finest: A*w scratch
    V_FC,        // finest: the prolonged correction (and natural-order staging)
    V_FR,        // finest: the residual between V-cycles (and natural-order staging)
    V_PSI,       // finest FP64: the solution
    V_SOURCE,    // finest FP64: the source
    V_P,         // finest FP64: the search direction
    V_ROLD,      // finest FP64: the previous residual (flexible beta)
    kRoles
};

// One case on one level, in value type T.
template <class T>
struct SegLevel
{
    k::Rows<T> rows;          // position-ordered rows (rows.n = cells)
    const int* posOf;         // cell -> position
    const int* posCell;       // position -> cell
    T* v[kRoles];
    int coarseSeg;            // this case's descriptor on the next level, -1 at its coarsest
    int nCoarse;
    const int* rStartP;       // the step to the next level: coarse position -> fine positions
    const int* rListP;
    const int* prolongP;      // fine position -> coarse position
    PcgScalars* scal;         // the case's PCG scalars
    int caseIdx;
    int pad;
    // the multicolour layout (hierarchy.cuh Colouring) and its FP32 values, once prepared
    const int* mcPos;
    const int* mcSlice;
    const int* mcCol;
    const float* mcVal;
    const float* mcDiag;
    const int* mcColourStart;  // [mcColours+1] rows of each colour
    int mcColours;
    int mcRows;
};

// Tiles of cells of some cases on one level: {descriptor, begin, end, the case's index in the list};
// a case's tiles are consecutive.
struct TileList
{
    DBuf<int4> tiles;
    DBuf<int> segOf;          // [nSeg] descriptor of each listed case
    DBuf<int> tileStart;      // [nSeg+1]
    int nTiles = 0;
    int nSeg = 0;
};

// The per-case perf the batch returns.
struct BatchPerf
{
    double initialResidual, finalResidual;
    int nIterations, pad;
};

struct BatchLevel
{
    TileList all;       // every case that has this level
    TileList up;        // the cases that go on to the next level (their cells here)
    TileList scale;     // the cases scaled here on the way up (two or more levels below)
    TileList down;      // the up cases, tiled over their next level's cells (restriction)
    // the Gauss-Seidel sweep of the up cases (level 0: all), one launch
    DBuf<k::GsArgs<double>> gs64;
    DBuf<k::GsArgs<float>> gs32;
    DBuf<int4> parts;
    int nParts = 0;
    int block = 0;
    size_t smem64 = 0, smem32 = 0;
    DBuf<unsigned> progress;
    size_t ticketAt = 0;  // the sweep launch's ticket counter: the word after the parts' progress lines
    std::vector<int4> hostParts;  // the parts table on the host
    // the exact form's smoothing calls by sweeps * 16 + value size: the cases whose level fits one CTA
    // run all their sweeps in one pipelined launch (pipe_kernels.cuh), the others the sweep above
    struct Pipe
    {
        int nSmall = 0;
        size_t smem = 0;
        DBuf<unsigned char> table;   // k::PipeArgs<T>[nSmall]
        DBuf<int> caseOf;            // [nSmall]
        DBuf<int4> partsBig;         // the parts of the cases that do not fit
        int nPartsBig = 0;
        bool use = false;            // measured faster than the sweep-by-sweep launches
        float msPipe = 0.f, msSweeps = 0.f;  // per smoothing call of every case, as measured
    };
    std::map<int, Pipe> pipe;
    std::vector<TileList> mc;  // per colour: the swept large cases' rows of that colour (multicolour form)
    DBuf<int> mcSmall;         // the swept small cases (descriptors): one block each sweeps them whole
    int nMcSmall = 0;
};

struct Batch
{
    cudaStream_t stream = nullptr;
    std::vector<Matrix*> cases;
    int maxLevels = 0;                      // the most coarse levels of any case
    std::vector<int> nLevelsOf;             // coarse levels of each case
    DBuf<SegLevel<double>> segD;            // every (case, level), level-major
    DBuf<SegLevel<float>> segF;
    std::vector<int> levelSeg0;             // first descriptor of each level
    std::vector<std::vector<int>> segOfCase;  // [case][level] -> descriptor
    std::vector<BatchLevel> lev;
    TileList coarsestTiles;                 // each case's cells on its coarsest level
    DBuf<k::CoarsestArgs<double>> coarsestArgs;  // [K] FP64 coarsest solve on (V_CORR, V_SRC)
    DBuf<k::DenseCase> denseCases;          // [K] the FP32 forms' direct coarsest solves (coarsestDirect)
    bool denseAll = false;                  // every case has its dense factor for the current values
    bool denseAny = false;                  // some case has its dense factor
    void prepareDense();
    unsigned long long layoutFingerprint() const;
    template <class T> void preparePipe(int lv, int nSweeps);
    void preparePipes(const b2g_controls& c);
    bool pipeOn = false;                    // the current solve takes the batched pipelined sweeps
    DBuf<int> active;                       // [K]
    DBuf<int> nActive;                      // [1]
    DBuf<int> err;
    DBuf<double> partial;                   // tile partials
    DBuf<double> sf64;                      // per listed case
    DBuf<float> partial32, sf32;
    DBuf<BatchPerf> perf;                   // [K]
    IterationGraph graph;
    std::vector<SegLevel<float>> hostF;    // host copy of segF
    bool mcReady = false;                   // the multicolour layouts are prepared
    bool multicolour = false;               // the current solve sweeps the FP32 V-cycle colour by colour
    bool denseNow = false;                  // the current solve takes the dense coarsest factors
    int eagerIterations = 0;                // iterations run without a graph (the first one)
    bool serial = false;
    long long launches = 0;

    Batch(std::vector<Matrix*> cases, cudaStream_t s);
    ~Batch();
    // every case: source and psi (natural cell order) in `memspace`, psi overwritten; perfs [K]
    void solve(const b2g_controls& c, const double* const* source, double* const* psi, int memspace,
               b2g_perf* perfs);

    template <class T> SegLevel<T>* segs();
    template <class T> void vcycle(const b2g_controls& c, int fresRole);
    template <class T> void smooth(int lv, int nSweeps);
    template <class T> void scale(int lv, const TileList& L, int field, int acf, int src, bool finest, int psi);
    void precondition(const b2g_controls& c);
    void reduce(int op, int a, int b, size_t member);
    void iteration(const b2g_controls& c);
    void prepareMulticolour();
    void buildMcLists(int lv, int threshold);
    std::vector<int> mcThreshold;           // per level: the tuned largest case swept by one block
    std::vector<float> mcSweepMs;           // per level: the tuned sweep's measured time
};

}  // namespace b2g
