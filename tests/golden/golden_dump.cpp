// golden_dump.cpp -- fixture generator (test infrastructure). Reads an OpenFOAM polyMesh with the
// reference's own mesh reader and geometry code (PrimitiveMesh::read, FvGeometry::build), so the
// face-area vectors in the fixture are bit-for-bit the ones the reference's agglomeration weighs.
// Built by `make -C oracle fixture` against the reference sources; run by make_golden.py.
//
// Output (little-endian binary): int32 nC, nIf, then owner[nIf], neighbour[nIf] (int32),
// Sf[3*nIf], magSf[nIf] (float64), int32 nPatches, then per patch: int32 nameLen, name bytes,
// int32 start, int32 size, faceCells[size] (int32).
#include "fv_geometry.cuh"
#include "primitive_mesh.cuh"

#include <cstdio>
#include <string>
#include <vector>

using namespace brae;

int main(int argc, char** argv)
{
    if (argc < 3)
    {
        std::fprintf(stderr, "usage: %s <polyMeshDir> <out.bin>\n", argv[0]);
        return 2;
    }
    PrimitiveMesh m;
    m.read(argv[1]);
    FvGeometry g;
    g.build(m);
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 1;
    const int nC = m.nCells();
    const int nIf = m.nInternalFaces();
    std::fwrite(&nC, 4, 1, f);
    std::fwrite(&nIf, 4, 1, f);
    std::fwrite(m.owner().data(), 4, static_cast<std::size_t>(nIf), f);
    std::fwrite(m.neighbour().data(), 4, static_cast<std::size_t>(nIf), f);
    for (int i = 0; i < nIf; ++i)
    {
        const vector s = g.Sf()[static_cast<std::size_t>(i)];
        const double v[3] = {s.x, s.y, s.z};
        std::fwrite(v, 8, 3, f);
    }
    std::fwrite(g.magSf().data(), 8, static_cast<std::size_t>(nIf), f);
    const int np = static_cast<int>(m.patches().size());
    std::fwrite(&np, 4, 1, f);
    for (const PatchInfo& p : m.patches())
    {
        const int len = static_cast<int>(p.name.size());
        std::fwrite(&len, 4, 1, f);
        std::fwrite(p.name.data(), 1, p.name.size(), f);
        std::fwrite(&p.start, 4, 1, f);
        std::fwrite(&p.size, 4, 1, f);
        for (int i = 0; i < p.size; ++i)
        {
            const int c = m.owner()[static_cast<std::size_t>(p.start + i)];
            std::fwrite(&c, 4, 1, f);
        }
    }
    std::fclose(f);
    return 0;
}
