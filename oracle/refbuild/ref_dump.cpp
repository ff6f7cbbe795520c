// Full-precision dump hook linked into the reference oracle (test
// infrastructure).  The reference prints forces and residuals with 4-6
// significant digits (codes/force/src/AeroForceTask.cpp:137-138,
// codes/residual/src/ResidualTask.cpp:169); parity at 1e-12 needs the raw
// fields.  After the run, when OFG_REF_DUMP names a file, this writes the
// first zone's fields as raw little-endian data:
//   int32 nCells, int32 nTCell, int32 nFields, then per field
//   char[16] name, int32 nEqu, double[nEqu][nTCell].
#include "Zone.h"
#include "ZoneState.h"
#include "UnsGrid.h"
#include "CellMesh.h"
#include "DataBase.h"
#include "HXArray.h"
#include "Force.h"
#include "AeroForceTask.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace ONEFLOW;

void OfgRefDump()
{
    const char *path = std::getenv("OFG_REF_DUMP");
    if (!path) return;
    ZoneState::zid = 0;
    UnsGrid *grid = Zone::GetUnsGrid();
    if (!grid) return;
    const char *names[] = {"q", "res", "dq", "timestep", "tempr", "visl", "vist", "turbq", "turbres", "turbdq", "dqdx", "dqdy", "dqdz", "limiter"};
    std::vector<std::pair<std::string, MRField *>> fields;
    // the turbulence fields exist only when the SA solver runs (looking up a
    // field name that was never allocated is not safe in the reference)
    bool turb = GetDataValue<int>("vismodel") >= 3;
    for (const char *n : names) {
        if (!turb && std::strncmp(n, "turb", 4) == 0) continue;
        MRField *f = GetFieldPointer<MRField>(grid, n);
        if (f) fields.push_back({n, f});
    }
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return;
    int nCells = grid->nCells;
    int nTCell = nCells + grid->nBFaces;
    // the wall distance (CellMesh::dist, one value per interior cell)
    RealField &dist = grid->cellMesh->dist;
    MRField distField(1, nTCell);
    for (int i = 0; i < nCells && i < (int)dist.size(); ++i) distField[0][i] = dist[i];
    if (turb) fields.push_back({"walldist", &distField});
    // the aerodynamic forces of the final state, by the reference's own
    // routines (AerodynamicForceTask::Run without its 4-digit file dump):
    // first 13 values of a one-row field "forces": total x y z, pressure
    // x y z, viscous x y z, CL, CD, CD_pres, CD_vis
    MRField forceField(1, nTCell);
    aeroForceInfo.Init();
    CalcAeroForce(0);
    aeroForceInfo.CollectForce();
    aeroForceInfo.CalcCoef();
    {
        AeroForce &t = aeroForceInfo.totalForce;
        double v[13] = {t.total.x, t.total.y, t.total.z, t.pres.x, t.pres.y, t.pres.z, t.vis.x, t.vis.y, t.vis.z,
                        aeroForceInfo.cl, aeroForceInfo.cd, aeroForceInfo.cd_pres, aeroForceInfo.cd_vis};
        for (int k = 0; k < 13 && k < nTCell; ++k) forceField[0][k] = v[k];
    }
    fields.push_back({"forces", &forceField});
    int nf = (int)fields.size();
    std::fwrite(&nCells, 4, 1, fp);
    std::fwrite(&nTCell, 4, 1, fp);
    std::fwrite(&nf, 4, 1, fp);
    for (auto &kv : fields) {
        char nm[16] = {0};
        std::strncpy(nm, kv.first.c_str(), 15);
        std::fwrite(nm, 1, 16, fp);
        MRField &f = *kv.second;
        int ne = (int)f.GetNEqu();
        std::fwrite(&ne, 4, 1, fp);
        for (int e = 0; e < ne; ++e) {
            std::vector<double> buf(nTCell, 0.0);
            int n = (int)f[e].size();
            for (int i = 0; i < nTCell && i < n; ++i) buf[i] = f[e][i];
            std::fwrite(buf.data(), 8, nTCell, fp);
        }
    }
    std::fclose(fp);
}
