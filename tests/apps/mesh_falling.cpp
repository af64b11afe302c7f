// Triangle-mesh particles read from an OBJ file falling into a box, written
// against the LSSolver call surface and its helper namespaces: OBJLoader::
// reads the mesh, LevelSetObject::TriangleMeshParticle builds its grid,
// SpherePacking::buildRegularInBox places the copies, BoxWall closes the box.
//
//   mesh_falling <outdir> <mesh.obj>
//
// Writes <outdir>/state.txt: one line per particle, position and velocity.
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "kernel/LSSolver.h"
#include "kernel/helper/LevelSetObjectGenerator.h"
#include "kernel/helper/OBJLoader.h"
#include "kernel/helper/SpherePackingGenerator.h"

struct Box : public LSSolver {
    explicit Box(const std::string& dir) : LSSolver(dir) {}
    bool writeState(const std::string& file)
    {
        const std::vector<double3>& x = getLSParticle().positionHostRef();
        const std::vector<double3>& v = getLSParticle().velocityHostRef();
        std::ofstream f(file);
        if (!f) return false;
        f.precision(17);
        for (size_t i = 0; i < x.size(); ++i)
            f << x[i].x << ' ' << x[i].y << ' ' << x[i].z << ' ' << v[i].x << ' ' << v[i].y << ' ' << v[i].z << '\n';
        return bool(f);
    }
};

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    const std::string out = argv[1];
    std::vector<double3> v;
    std::vector<int3> f;
    if (!OBJLoader::loadOBJMesh(argv[2], v, f, argc, argv)) return 1;
    LevelSetObject::TriangleMeshParticle mesh;
    mesh.setMesh(v, f);
    mesh.buildGridByResolution(30);
    if (!mesh.isGridBuilt()) return 1;

    const double3 lo = make_double3(0.0, 0.0, 0.0), hi = make_double3(1.0, 1.0, 2.0);
    const double d = length(mesh.boundingBoxMax() - mesh.boundingBoxMin());
    const SpherePacking::Pack pack = SpherePacking::buildRegularInBox(lo, hi, 0.5 * d);

    std::filesystem::create_directories(out);
    Box box(out);
    box.addParticleMaterial(6.0e5, 1.8e5, 0.5, 0.8);
    std::vector<double3> zero(pack.centers.size(), make_double3(0, 0, 0));
    std::vector<quaternion> q(pack.centers.size(), make_quaternion(1, 0, 0, 0));
    const LevelSetObject::GridInfo& g = mesh.gridInfo();
    box.addParticleCluster(pack.centers, zero, zero, q, 0, 1000.0, g.gridOrigin, g.gridNodeSpacing, g.gridNodeSize,
                           g.gridNodeSignedDistance, mesh.vertexPosition(), mesh.triangleVertexIndex());

    LevelSetObject::BoxWall wall;
    wall.setParams(hi.x - lo.x, hi.y - lo.y, hi.z - lo.z);
    wall.buildGridByResolution(40);
    const LevelSetObject::GridInfo& wg = wall.gridInfo();
    box.addWallMaterial(0.5, 0.8);
    box.addWallGeometry(wg.gridOrigin, wg.gridNodeSpacing, wg.gridNodeSize, wg.gridNodeSignedDistance,
                        wall.vertexPosition(), wall.triangleVertexIndex());
    box.addWall(0.5 * (lo + hi), make_double3(0, 0, 0), make_double3(0, 0, 0), make_quaternion(1, 0, 0, 0), 0, 0);
    box.solve(lo, hi, make_double3(0.0, 0.0, -9.81), 1.0e-4, 0.5, 2, argc, argv);
    if (!box.writeState(out + "/state.txt")) return 1;
    std::printf("particles %zu\n", pack.centers.size());
    return 0;
}
