// OBJLoader::loadOBJMesh -- reads the vertices and faces of a Wavefront OBJ
// file into the arrays TriangleMeshParticle::setMesh takes.  The entry point
// keeps the reference's name and argument list (kernel/helper/OBJLoader.h,
// called as in apps/tutorial/LSParticleFalling.cpp:57); the parser is this
// project's own.
//
// Accepted input:
//   * "v x y z" lines (vertices) and "f a b c ..." lines (faces); every other
//     line ("vn", "vt", "o", "g", "usemtl", comments after '#') is skipped;
//   * a face corner is "i", "i/t", "i//n" or "i/t/n"; only i is used;
//     i > 0 counts from the first vertex (1-based), i < 0 back from the last
//     vertex read so far;
//   * a polygon of k corners becomes the k - 2 triangles of a fan from its
//     first corner.
// A relative file name is taken from the running executable's directory
// (argv[0]); an absolute one as it is.  On a malformed file the arrays are
// left empty, a message naming the line goes to std::cerr, and the call
// returns false.  With verbose, the counts go to std::cout.
#pragma once
#include <cerrno>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include <vector_functions.h>
#include <vector_types.h>

namespace OBJLoader
{
namespace detail
{

// A read position within one line.
struct Cursor {
    const char* p;
    const char* end;

    static bool space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f'; }
    void skip_space()
    {
        while (p < end && space(*p)) ++p;
    }
    bool at_end()
    {
        skip_space();
        return p >= end || *p == '#';
    }
    // the next whitespace-delimited word
    std::string word()
    {
        skip_space();
        const char* a = p;
        while (p < end && !space(*p)) ++p;
        return std::string(a, p);
    }
    bool number(double& out)
    {
        const std::string w = word();
        if (w.empty()) return false;
        char* stop = nullptr;
        errno = 0;
        out = std::strtod(w.c_str(), &stop);
        return stop == w.c_str() + w.size() && errno != ERANGE;
    }
};

// the vertex part of a face corner, as a 0-based index; false when the
// corner is malformed or names no vertex read so far
inline bool corner_index(const std::string& corner, long long nvert, int& out)
{
    const std::string head = corner.substr(0, corner.find('/'));
    if (head.empty()) return false;
    char* stop = nullptr;
    errno = 0;
    const long long i = std::strtoll(head.c_str(), &stop, 10);
    if (stop != head.c_str() + head.size() || errno == ERANGE || i == 0) return false;
    const long long z = i > 0 ? i - 1 : nvert + i;
    if (z < 0 || z >= nvert) return false;
    out = static_cast<int>(z);
    return true;
}

inline std::filesystem::path locate(const std::string& filename, int argc, char** argv)
{
    const std::filesystem::path name(filename);
    if (name.is_absolute()) return name;
    std::filesystem::path base = std::filesystem::current_path();
    if (argc > 0 && argv != nullptr && argv[0] != nullptr) {
        std::error_code ec;
        const std::filesystem::path exe = std::filesystem::weakly_canonical(std::filesystem::absolute(argv[0]), ec);
        if (!ec) base = exe.parent_path();
    }
    return base / name;
}

// parses the stream; on failure returns false with the line number and reason
inline bool parse(std::istream& in, std::vector<double3>& vertices, std::vector<int3>& faces, std::size_t& line_no,
                  std::string& why)
{
    std::string line;
    std::vector<int> poly;
    line_no = 0;
    while (std::getline(in, line)) {
        ++line_no;
        Cursor c{line.data(), line.data() + line.size()};
        if (c.at_end()) continue;
        const std::string tag = c.word();
        if (tag == "v") {
            double x, y, z;
            if (!c.number(x) || !c.number(y) || !c.number(z)) {
                why = "vertex needs three numbers";
                return false;
            }
            vertices.push_back(make_double3(x, y, z));
        } else if (tag == "f") {
            poly.clear();
            while (!c.at_end()) {
                int id = 0;
                const std::string corner = c.word();
                if (!corner_index(corner, static_cast<long long>(vertices.size()), id)) {
                    why = "bad face corner '" + corner + "'";
                    return false;
                }
                poly.push_back(id);
            }
            if (poly.size() < 3) {
                why = "face with fewer than three corners";
                return false;
            }
            for (std::size_t k = 2; k < poly.size(); ++k) faces.push_back(make_int3(poly[0], poly[k - 1], poly[k]));
        }
    }
    return true;
}

}  // namespace detail

inline bool loadOBJMesh(const std::string& filename, std::vector<double3>& vertices, std::vector<int3>& faces,
                        const int argc, char** argv, const bool verbose = true)
{
    vertices.clear();
    faces.clear();
    const std::filesystem::path path = detail::locate(filename, argc, argv);
    std::ifstream in(path);
    if (!in) {
        std::cerr << "OBJLoader: cannot open " << path.string() << std::endl;
        return false;
    }
    std::size_t line_no = 0;
    std::string why;
    if (!detail::parse(in, vertices, faces, line_no, why)) {
        std::cerr << "OBJLoader: " << path.string() << ":" << line_no << ": " << why << std::endl;
        vertices.clear();
        faces.clear();
        return false;
    }
    if (verbose)
        std::cout << "OBJLoader: " << path.string() << ": " << vertices.size() << " vertices, " << faces.size()
                  << " triangles" << std::endl;
    return true;
}

}  // namespace OBJLoader
