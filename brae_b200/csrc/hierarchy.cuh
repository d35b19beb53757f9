// hierarchy.cuh -- the per-mesh GAMG hierarchy held on the device: each level's LDU addressing
// with the derived layouts every kernel reads, and each level step's restriction maps.
#pragma once

#include <atomic>

#include "b2g_common.cuh"

#include <map>
#include <memory>

namespace b2g {

// The sweep order of one level and its Gauss-Seidel schedule (gs_kernels.cuh). Cells are split into
// `nParts` contiguous index ranges; each part lists its cells by (depth, cell), depth being the cell's
// level in the forward DAG (a cell depends on the owners of the faces it is the neighbour of).
// "Positions" index that (part, depth, cell) order, and EVERY device vector of the level is stored in
// position order. A part's positions are cut into chunks of at most maxCells cells of one depth.
struct GsSchedule
{
    int nParts = 0;
    int maxDepth = 0;
    int nChunks = 0;
    int maxCells = 0;          // chunk cell capacity == the kernel's compute threads
    int maxEnt = 0;            // chunk ELL entry capacity
    int maxGat = 0;            // chunk gather capacity (per stage in the sweep's value table)
    int ahead = 0;             // window extents the entry codes assume (gsWindowExtents)
    int behind = 0;
    int nPadded = 0;           // position count rounded up to the window fill block
    int nAlloc = 0;            // allocation length of every position-ordered vector of the level
    long long nEll = 0;        // ELL entries (whole 32-cell slices, padding included)
    long long nGather = 0;     // gathered values over all chunks
    long long blobBytes64 = 0; // the chunks' blobs (gs_kernels.cuh) in FP64 and in FP32
    long long blobBytes32 = 0;
    DBuf<int> depth;           // [nCells] by cell
    DBuf<int> partChunkStart;  // [nParts+1]
    DBuf<int> partPosStart;    // [nParts+1] (a part's positions are its cell range)
    DBuf<int> chunkRec;        // [nChunks][12] (gs_kernels.cuh ChunkRec)
    DBuf<int> upStart;         // [nParts+1] upstream parts of each part
    DBuf<int> upList;
    DBuf<int> hasDown;         // [nParts] 1 if another part reads this part's new values
    DBuf<int> posCell;         // [nCells] cell at each position
    DBuf<int> posOf;           // [nCells] position of each cell
    DBuf<int> posRow;          // [nCells+1 (+pad)] CSR entry offsets in position order
    DBuf<int> entColPos;       // [2*nFaces] CSR: the other cell's position per entry
    DBuf<int> entFacePos;      // [2*nFaces] CSR: face of each entry
    DBuf<unsigned> posEnt;     // [nCells (+pad)] sweep row descriptor: slice width << 24 | chunk-relative base
    DBuf<unsigned short> gsCode;  // [nEll] sweep entry codes: value-table indices (gs_kernels.cuh)
    DBuf<int> gsEntFace;       // [nEll] face of each sweep entry, -1 for padding
    DBuf<int> gatSrc;          // [nGather] position of each gathered value
    DBuf<unsigned> progress;   // [nParts][kProgressStride] per-part progress words, one L2 line each
                               // (reset before each launch)
    // an item schedule (items.cu) of `items` sweeps pipelined: "positions" index (sweep, cell) items,
    // and itemStore[i] is the psi position item i writes
    int items = 0;
    DBuf<int> itemStore;
    // the position-order rows in sliced ELL (ldu_kernels.cuh Rows), on levels of at least
    // kEllMinCells cells: per 32-position slice its entry base [nCells/32 + 1], per entry the column
    // position (-1 past the row's end) and the CSR entry it copies (-1 there)
    long long nEllEnt = 0;
    DBuf<int> ellBase, ellCol, ellEnt;
    // the finest level's: per ELL entry the coarse position its column is prolonged from (-1 past the
    // row's end), so that the correction scaling reads the coarse correction with one gather
    DBuf<int> ellColCoarse;
};

// the smallest level that gets the sliced ELL copy of its rows
constexpr int kEllMinCells = 65536;

// the multi-part sweep's part rule for meshes built from now on: one part per this many cells of a
// level's average depth (b2g_set_part_cells)
extern std::atomic<int> g_partCells;

// One smoothing call's sweeps of a level in one pipelined launch (pipe_kernels.cuh), for a given
// sweep count: the combined steps of every (sweep, cell) item, the cells split into `ranks`
// contiguous ranges held in the shared memory of one CTA each (one cluster when ranks > 1), or, in
// the grid form, owned by one of `ranks` resident CTAs with psi in global memory.
struct PipeSchedule
{
    int sweeps = 0;
    int ranks = 0;
    int nSteps = 0;
    int maxLocal = 0;           // shared-memory slots per rank (0 in the grid form)
    DBuf<int> stepStart;        // [ranks][nSteps + 1] item ranges
    DBuf<int4> item;            // [sweeps * nCells] {position, value slot, first entry, end entry}
    DBuf<unsigned> entAddr;     // [2 * nFaces] per position-order row entry: rank << 24 | slot
    DBuf<int> localPos;         // [ranks][maxLocal] position of each slot
    DBuf<int> localCount;       // [ranks]
    // the grid form: a row's value slot is its position and it reads psi at the level's columns; each
    // rank waits for its neighbour ranks only
    bool grid = false;
    DBuf<int> nbrStart;         // [ranks + 1]
    DBuf<int> nbrList;
    DBuf<unsigned> progress;    // [ranks][kProgressStride]
};

// The dynamic shared memory of a pipelined launch in values of valueBytes (pipe.cu): the rank's
// slots in the shared-memory forms, the rank's step table in the grid form.
size_t pipeSmemBytes(const PipeSchedule& P, size_t valueBytes);


// The choice for one (level, sweep count, value type), by measurement (Matrix::ensurePipe): the
// pipelined launch with the fastest shape (shared memory on 1-16 CTAs, or the grid form), the item
// schedule, or the sweep-by-sweep launches when those are faster.
struct PipeChoice
{
    int mode = 0;                        // 0 sweep by sweep, 1 the pipelined launch, 2 items
    std::unique_ptr<PipeSchedule> sched; // mode 1 (shared memory, or the grid form)
    std::unique_ptr<GsSchedule> items;   // mode 2: the multi-part sweep over (sweep, cell) items
    float msPipe = 0.f;   // per smoothing call, the best shared-memory shape (0: none fits)
    float msItems = 0.f;  // per smoothing call, the item schedule (0: not built)
    float msSweeps = 0.f; // per smoothing call, sweep by sweep
    float msGrid = 0.f;   // per smoothing call, the best grid form (0: not tried)
};

struct LevelAddr;
// The item schedule of L for S sweeps pipelined in one launch (items.cu), or null when the level has
// one part or exceeds the schedule's limits.
std::unique_ptr<GsSchedule> buildGsItems(const LevelAddr& L, int S, cudaStream_t s);
// L's one-CTA pipelined schedule for S sweeps in values of valueBytes (pipe.cu), built once and kept on
// the level; null when the level's psi does not fit one CTA's shared memory.
const PipeSchedule* pipeOneCta(LevelAddr& L, int S, size_t valueBytes, cudaStream_t s);

// A colouring of one level for the multicolour sweep of the FP32 V-cycle: no two cells of one colour
// share a face, so a colour's cells are updated in parallel. Rows are the level's cells colour by
// colour (ascending cell within a colour), each colour padded to whole 32-row slices, entries in
// sliced ELL (entry q of the row in lane l of slice s at sliceBase[s] + 32*q + l); padding rows have
// pos -1, padding entries face -1. Within a colour, rows follow the level's position order.
struct Colouring
{
    int nColours = 0;
    std::vector<int> colourStart;  // [nColours+1] rows (host)
    DBuf<int> colourStartD;        // the same on the device
    int nRows = 0;
    long long nEnt = 0;
    DBuf<int> pos;                 // [nRows] position of each row's cell
    DBuf<int> sliceBase;           // [nRows/32 + 1]
    DBuf<int> col;                 // [nEnt] the other cell's position
    DBuf<int> face;                // [nEnt] the face, -1 for padding
    // the sweep's launch shape, chosen by measurement (Matrix::tuneMulticolour): one block sweeping
    // the whole level, one thread-block cluster of `cluster` CTAs sweeping it (cluster > 0), or one
    // launch per colour of `block` threads per block
    bool tuned = false;
    bool fused = false;
    int cluster = 0;
    int block = 256;
    float msPerSweep = 0.f;
    // per smoothing call of nSweeps sweeps (key nSweeps * 2 + symmetric): the pipelined shared-memory
    // launch (pipe.cu) whose steps are the colours, kept where it measured faster than the shape above
    struct Pipe
    {
        std::unique_ptr<PipeSchedule> sched;
        bool use = false;
        float msPipe = 0.f, msColours = 0.f;  // per smoothing call, as measured
    };
    std::map<int, Pipe> pipe;
};

// The coupled (cyclic) pair of one level (pair.cu, b2g_mesh_set_pair): its faces, each once from
// its own side, as (own, nbr) cells of this level in face order -- the finest level's as the coupled
// patches list them (gamgLevel0Interface, GAMG:440-470), a coarse level's agglomerated from the finer
// one on the coarse cell pair (GAMG:497-524). By position, the pair entries of each row in face order.
struct PairLevel
{
    int nFaces = 0;
    std::vector<int> own, nbr;  // host, cells of this level
    DBuf<int> start;            // [nCells+1] position -> its entries (the faces the cell owns)
    DBuf<int> col;              // [nFaces] per entry: the neighbour's position
    DBuf<int> face;             // [nFaces] per entry: the pair face
    DBuf<int> fStart;           // coarse levels: [nFaces+1] this level's face -> the finer level's
    DBuf<int> fList;            //   faces that merged into it, ascending (the coefficient sum's order)
};

// One level's addressing and its derived layouts (built once per hierarchy).
struct LevelAddr
{
    int nCells = 0;
    int nFaces = 0;
    DBuf<int> lower;        // [nFaces] owner
    DBuf<int> upper;        // [nFaces] neighbour
    DBuf<int> ownStart;     // [nCells+1] owned-face ranges (faces are sorted by owner)
    DBuf<int> losortStart;  // [nCells+1]
    DBuf<int> losort;       // [nFaces] faces ordered by neighbour cell, ascending face within a cell
    // Cell-ordered rows in the reference's per-cell accumulation order: the faces the cell is the
    // neighbour of (ascending face), then the faces it owns (ascending face). Amul, the residual,
    // normFactor's row sums and the Gauss-Seidel gather all walk a cell's terms in this order.
    DBuf<int> rowStart;     // [nCells+1] = losortStart + ownStart
    DBuf<int> col;          // [2*nFaces] the other cell
    DBuf<int> entFace;      // [2*nFaces] the face
    GsSchedule gs;
    Colouring mc;           // built on first use (buildColouring)
    // The backward walk of symGaussSeidel as a forward sweep (built on first use, buildReversedLevel):
    // cells renumbered n-1-c, each row holding only the cell's own faces (it owns them in this level)
    // in ascending face order, tagged with this level's face ids; its own schedule and positions.
    std::unique_ptr<LevelAddr> rev;
    DBuf<int> revPos;       // [nCells] this level's position -> the reversed level's position
    // DIC's substitutions as forward sweeps (built on first use): the forward one on a level whose
    // rows hold only the faces the cell is the neighbour of (ascending), the backward one on a
    // reversed level whose rows hold the cell's own faces in DESCENDING face order
    std::unique_ptr<LevelAddr> lowerOnly;
    DBuf<int> lowerPos;
    std::unique_ptr<LevelAddr> revDesc;
    DBuf<int> revDescPos;
    PairLevel pair;         // the coupled pair, if the mesh carries one (nFaces 0 otherwise)
    // pipelined smoothing calls, keyed by sweeps * 16 + the value size (built on first use)
    std::map<int, PipeChoice> pipe;
    // the one-CTA pipelined schedule by the same key (the batched form's; null: the level does not fit)
    std::map<int, std::unique_ptr<PipeSchedule>> pipeOne;
    // The one-block resident Gauss-Seidel sweep of a small one-part level (solver.cu gsResident),
    // built on first use: the part's positions run by depth, depth d's are [start[d], start[d+1]).
    struct Resident
    {
        bool built = false;
        bool ok = false;     // the level qualifies (one part, small enough, positions by depth)
        int nDepth = 0;
        int block = 0;       // threads: the widest depth rounded up to a warp, 64..256
        DBuf<int> start;     // [nDepth+1]
    } resident;
};

// Level step i -> i+1 (GamgAgglomeration's restrictAddressing / faceRestrictAddressing /
// faceFlipMap) with the inverse lists the gather kernels need.
struct Step
{
    int nFine = 0, nCoarse = 0, nFineFaces = 0, nCoarseFaces = 0;
    DBuf<int> restrictAddr;   // [nFine] fine cell -> coarse cell
    DBuf<int> faceRestrict;   // [nFineFaces] >= 0 coarse face, else -(coarse cell + 1)
    DBuf<int8_t> flip;        // [nFineFaces]
    DBuf<int> cellStart;      // [nCoarse+1] coarse cell -> its fine cells, ascending
    DBuf<int> cellList;       // [nFine]
    DBuf<int> intStart;       // [nCoarse+1] coarse cell -> fine faces inside it, ascending
    DBuf<int> intList;
    DBuf<int> faceBeg;        // [nCoarseFaces] coarse face -> fine faces [faceBeg, faceEnd) of faceList
    DBuf<int> faceEnd;
    DBuf<int> faceList;       // fine faces, grouped by coarse face, ascending within a group
    // the same maps on the two levels' position orders
    DBuf<int> rStartP;        // [nCoarse+1] coarse position -> its fine positions in rListP
    DBuf<int> rListP;         // [nFine] fine positions, in ascending fine-cell order per coarse cell
    DBuf<int> prolongP;       // [nFine] fine position -> coarse position
};

struct Mesh
{
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<LevelAddr> lev;  // [0] the mesh, [i] coarse level i
    std::vector<Step> step;      // [i] level i -> i+1
    float buildMs = 0.f;
    bool hasPair = false;        // b2g_mesh_set_pair was called (every level's PairLevel is built)
    int nLevels() const { return static_cast<int>(step.size()); }
};

// Builds the derived layouts of `L` from its lower/upper (already on the device). Validates the
// upper-triangular order (faces sorted by owner, owner < neighbour).
void buildLevelLayouts(LevelAddr& L, cudaStream_t s);
// The sweep order and Gauss-Seidel schedule of `L` (depths, parts, positions, chunks, codes).
void buildGsSchedule(LevelAddr& L, cudaStream_t s);
// The multicolour layout of `L` (greedy colouring in cell order; a structured hex level gets the two
// colours of a checkerboard). Needs the level's schedule (positions).
void buildColouring(LevelAddr& L, cudaStream_t s);
// The reversed level of `L` for symGaussSeidel's backward walk (needs L's schedule); with
// `descending`, the one for DIC's backward substitution (L.revDesc).
void buildReversedLevel(LevelAddr& L, cudaStream_t s, bool descending = false);
// The lower-only level of `L` for DIC's forward substitution (L.lowerOnly).
void buildLowerLevel(LevelAddr& L, cudaStream_t s);
// The position-ordered restriction and prolongation maps of step `i` (both levels scheduled).
void buildStepMaps(Mesh& M, int i);
// The whole agglomeration (faceAreaPairGamgAgglomeration) from device arrays.
void buildHierarchy(Mesh& M, const double* dSf, const double* dMagSf, int nCellsInCoarsestLevel,
                    int* forward);

// The same hierarchy from known restriction maps (a cached agglomeration): the pairing passes are
// skipped; maps[i] is step i's restrictAddr (host), nCoarse[i] its coarse cell count.
void buildHierarchyFromMaps(Mesh& M, const double* dSf, const double* dMagSf,
                            const std::vector<std::vector<int>>& maps, const std::vector<int>& nCoarse);

// The coupled pair on every level (pair.cu): the finest level's nFaces faces (host cells own/nbr),
// each coarse level's agglomerated from the finer one.
void buildPair(Mesh& M, int nFaces, const int* own, const int* nbr);

// Exclusive scan helper (n+1 outputs: out[0] = 0 ... out[n] = total); returns the total.
long long exclusiveScan(const int* in, int* out, int n, cudaStream_t s);
// Stable radix sort of (key, value) pairs; keys are unsigned, sorted on the low `bits` bits.
void sortPairs(const unsigned* kin, unsigned* kout, const int* vin, int* vout, int n, int bits,
               cudaStream_t s);
void sortPairs64(const unsigned long long* kin, unsigned long long* kout, const int* vin,
                 int* vout, int n, int bits, cudaStream_t s);
// Histogram of keys in [0, nBins) and its exclusive scan into start[nBins+1].
void countingStarts(const int* keys, int n, int nBins, int* start, cudaStream_t s);

}  // namespace b2g
