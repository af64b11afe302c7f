// helpers_dump -- test infrastructure, not part of the product.
//
// Runs the level-set shape, sphere-packing and OBJ helpers on the cases read
// from standard input and writes every result to a binary file, so that two
// builds of this one source can be compared:
//   * against the reference's headers (kernel/helper/*.h, compiled where they
//     lie by `make -C oracle helpers`), producing the golden fixtures;
//   * against this library's drop-in headers (fundem_b200/kernel/helper/*.h),
//     whose grids are evaluated on the GPU.
//
//   helpers_dump OUT [nogrid|host] < cases.txt
//
// `host` builds every shape as a class derived from the named one; the
// reference is unaffected, while this library then evaluates the grid on the
// host through the virtual implicit function instead of on the GPU.
//
// One case per line (lengths in any unit):
//   SE name rx ry rz ee en subdivision res pad     Superellipsoid
//   SP name radius points res pad                  Sphere
//   BX name lx ly lz res pad                       BoxWall
//   CY name ax ay az bx by bz radius nc na res pad CylinderWall
//   MS name file.obj positive_inside res pad       OBJ mesh -> TriangleMeshParticle
//   PR name x0 y0 z0 x1 y1 z1 r                    buildRegularInBox
//   PH name x0 y0 z0 x1 y1 z1 r                    buildHexInBox
//   PB name x0 y0 z0 x1 y1 z1 n rmin rmax seed attempts   random packing in a box
//   PC name ax ay az bx by bz R n rmin rmax seed attempts  random packing in a cylinder
//   QR name x0 y0 z0 x1 y1 z1 r                    SpherePack::buildRegularInBox (kernel/Packing.h)
//   QH name x0 y0 z0 x1 y1 z1 r                    SpherePack::buildHexInBox
//   QB name x0 y0 z0 x1 y1 z1 n rmin rmax seed attempts   SpherePack::buildNonOverlappingInBox_LargeFirst
// Shapes write name/vertices, name/triangles and, unless `nogrid`, the grid of
// buildGridByResolution(res, pad): name/origin, name/size, name/spacing,
// name/sdf.  Packings write name/centers and name/radii.
//
// Record format: int32 name length, name bytes, int32 type (0 float64,
// 1 int32), int64 element count, the elements.
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "kernel/helper/LevelSetObjectGenerator.h"
#include "kernel/helper/OBJLoader.h"
#include "kernel/helper/SpherePackingGenerator.h"
#include "kernel/Packing.h"

namespace {

FILE* g_out = nullptr;

void put(const std::string& name, int type, const void* data, int64_t count)
{
    const int32_t n = (int32_t)name.size();
    std::fwrite(&n, 4, 1, g_out);
    std::fwrite(name.data(), 1, n, g_out);
    std::fwrite(&type, 4, 1, g_out);
    std::fwrite(&count, 8, 1, g_out);
    if (count > 0) std::fwrite(data, type == 0 ? 8 : 4, (size_t)count, g_out);
}

void put_d(const std::string& name, const std::vector<double>& v) { put(name, 0, v.data(), (int64_t)v.size()); }
void put_i(const std::string& name, const std::vector<int>& v) { put(name, 1, v.data(), (int64_t)v.size()); }

void put_mesh(const std::string& name, const LevelSetObject::TriangleMeshParticle& s)
{
    std::vector<double> v;
    for (const double3& p : s.vertexPosition()) v.insert(v.end(), {p.x, p.y, p.z});
    std::vector<int> t;
    for (const int3& f : s.triangleVertexIndex()) t.insert(t.end(), {f.x, f.y, f.z});
    put_d(name + "/vertices", v);
    put_i(name + "/triangles", t);
}

void put_grid(const std::string& name, LevelSetObject::Base& s, int res, int pad, bool grid)
{
    if (!grid) return;
    s.buildGridByResolution(res, pad);
    const LevelSetObject::GridInfo& g = s.gridInfo();
    put_d(name + "/origin", {g.gridOrigin.x, g.gridOrigin.y, g.gridOrigin.z});
    put_i(name + "/size", {g.gridNodeSize.x, g.gridNodeSize.y, g.gridNodeSize.z});
    put_d(name + "/spacing", {g.gridNodeSpacing});
    put_d(name + "/sdf", g.gridNodeSignedDistance);
}

// the named class itself, or a class derived from it that adds nothing
template <class S>
using Plain = S;
template <class S>
struct Derived : S {
};

void put_pack(const std::string& name, const SpherePacking::Pack& p)
{
    std::vector<double> c;
    for (const double3& x : p.centers) c.insert(c.end(), {x.x, x.y, x.z});
    put_d(name + "/centers", c);
    put_d(name + "/radii", p.radii);
}

template <template <class> class W>
int run(bool grid, int argc, char** argv)
{
    std::string line;
    while (std::getline(std::cin, line)) {
        std::istringstream in(line);
        std::string kind, name;
        if (!(in >> kind >> name)) continue;
        if (kind == "SE") {
            double rx, ry, rz, ee, en;
            int sub, res, pad;
            in >> rx >> ry >> rz >> ee >> en >> sub >> res >> pad;
            W<LevelSetObject::Superellipsoid> s;
            s.setParams(rx, ry, rz, ee, en, sub);
            put_mesh(name, s);
            put_grid(name, s, res, pad, grid);
        } else if (kind == "SP") {
            double r;
            size_t points;
            int res, pad;
            in >> r >> points >> res >> pad;
            W<LevelSetObject::Sphere> s;
            s.setParams(r, points);
            put_mesh(name, s);
            put_grid(name, s, res, pad, grid);
        } else if (kind == "BX") {
            double lx, ly, lz;
            int res, pad;
            in >> lx >> ly >> lz >> res >> pad;
            W<LevelSetObject::BoxWall> s;
            s.setParams(lx, ly, lz);
            put_mesh(name, s);
            put_grid(name, s, res, pad, grid);
        } else if (kind == "CY") {
            double ax, ay, az, bx, by, bz, r;
            int nc, na, res, pad;
            in >> ax >> ay >> az >> bx >> by >> bz >> r >> nc >> na >> res >> pad;
            W<LevelSetObject::CylinderWall> s;
            s.setParams(make_double3(ax, ay, az), make_double3(bx, by, bz), r, nc, na);
            put_mesh(name, s);
            put_grid(name, s, res, pad, grid);
        } else if (kind == "MS") {
            std::string file;
            int flip, res, pad;
            in >> file >> flip >> res >> pad;
            std::vector<double3> v;
            std::vector<int3> f;
            if (!OBJLoader::loadOBJMesh(file, v, f, argc, argv, false)) return 1;
            W<LevelSetObject::TriangleMeshParticle> s;
            s.setMesh(v, f);
            s.setLevelSetPositiveInside(flip != 0);
            put_mesh(name, s);
            put_grid(name, s, res, pad, grid);
        } else if (kind == "PR" || kind == "PH") {
            double3 a, b;
            double r;
            in >> a.x >> a.y >> a.z >> b.x >> b.y >> b.z >> r;
            put_pack(name, kind == "PR" ? SpherePacking::buildRegularInBox(a, b, r)
                                        : SpherePacking::buildHexInBox(a, b, r));
        } else if (kind == "PB" || kind == "PC") {
            double3 a, b;
            double R = 0.0, rmin, rmax;
            int n, attempts;
            uint32_t seed;
            in >> a.x >> a.y >> a.z >> b.x >> b.y >> b.z;
            if (kind == "PC") in >> R;
            in >> n >> rmin >> rmax >> seed >> attempts;
            put_pack(name, kind == "PB"
                               ? SpherePacking::buildNonOverlappingInBox_LargeFirst(a, b, n, rmin, rmax, seed, attempts)
                               : SpherePacking::buildNonOverlappingInCylinder_LargeFirst(a, b, R, n, rmin, rmax, seed,
                                                                                         attempts));
        } else if (kind == "QR" || kind == "QH" || kind == "QB") {
            double3 a, b;
            in >> a.x >> a.y >> a.z >> b.x >> b.y >> b.z;
            SpherePack p;
            if (kind == "QB") {
                double rmin, rmax;
                int n, attempts;
                uint32_t seed;
                in >> n >> rmin >> rmax >> seed >> attempts;
                p.buildNonOverlappingInBox_LargeFirst(a, b, n, rmin, rmax, seed, attempts);
            } else {
                double r;
                in >> r;
                if (kind == "QR") p.buildRegularInBox(a, b, r);
                else p.buildHexInBox(a, b, r);
            }
            SpherePacking::Pack q;
            q.centers = p.centers;
            q.radii = p.radii;
            put_pack(name, q);
        } else {
            std::cerr << "helpers_dump: unknown case kind " << kind << std::endl;
            return 2;
        }
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: helpers_dump OUT [nogrid|host] < cases.txt" << std::endl;
        return 2;
    }
    const std::string mode = argc > 2 ? argv[2] : "";
    g_out = std::fopen(argv[1], "wb");
    if (!g_out) return 2;
    const int rc = mode == "host" ? run<Derived>(true, argc, argv) : run<Plain>(mode != "nogrid", argc, argv);
    std::fclose(g_out);
    return rc;
}
