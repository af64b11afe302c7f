// OBJLoader:: -- reads the vertices and faces of a Wavefront OBJ file into the
// arrays TriangleMeshParticle::setMesh takes, with the names and behaviour of
// the reference's kernel/helper/OBJLoader.h: relative file names resolve
// against the executable's directory, face tokens may carry /vt/vn parts,
// negative indices count back from the last vertex, polygons become triangle
// fans from their first corner, and a malformed file yields empty arrays and
// false.
#pragma once
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <vector_functions.h>
#include <vector_types.h>

// directory of the running executable, from argv[0] (OBJLoader.h:22-33)
inline std::filesystem::path getExecutableDirectory(const char* argv0)
{
    if (argv0 == nullptr) return std::filesystem::current_path();
    std::filesystem::path exe(argv0);
    if (exe.is_relative()) exe = std::filesystem::absolute(exe);
    return std::filesystem::weakly_canonical(exe).parent_path();
}

// an absolute name is kept; a relative one is taken from the executable's directory
inline std::string resolvePathFromExecutable(const std::string& filename, const char* argv0)
{
    const std::filesystem::path p(filename);
    if (p.is_absolute()) return p.string();
    return (getExecutableDirectory(argv0) / p).string();
}

namespace OBJLoader
{

inline std::string trim(const std::string& s)
{
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

inline bool startsWith(const std::string& s, const std::string& prefix)
{
    return s.compare(0, prefix.size(), prefix) == 0;
}

// the vertex index of a face token "v", "v/vt", "v//vn" or "v/vt/vn"
inline int parseOBJVertexIndex(const std::string& token)
{
    if (token.empty()) throw std::runtime_error("Empty face token in OBJ.");
    const std::string head = token.substr(0, token.find('/'));
    if (head.empty()) throw std::runtime_error("Invalid OBJ face token: " + token);
    return std::stoi(head);
}

// 1-based from the start, or negative from the end of the vertices read so far
inline int convertOBJIndexToZeroBased(const int objIndex, const int numVertices)
{
    if (objIndex > 0) return objIndex - 1;
    if (objIndex < 0) return numVertices + objIndex;
    throw std::runtime_error("OBJ index cannot be zero.");
}

inline bool loadOBJMesh(const std::string& filename, std::vector<double3>& vertices, std::vector<int3>& faces,
                        const int argc, char** argv, const bool verbose = true)
{
    vertices.clear();
    faces.clear();
    const char* argv0 = (argc > 0 && argv != nullptr) ? argv[0] : nullptr;
    const std::string path = resolvePathFromExecutable(filename, argv0);
    std::ifstream in(path);
    if (!in.is_open()) {
        std::cerr << "[OBJLoader] Failed to open file: " << path << std::endl;
        return false;
    }
    std::string line;
    size_t lineNumber = 0;
    try {
        while (std::getline(in, line)) {
            ++lineNumber;
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            if (startsWith(line, "v ")) {
                std::istringstream ss(line.substr(2));
                double x, y, z;
                ss >> x >> y >> z;
                if (ss.fail()) throw std::runtime_error("Failed to parse vertex at line " + std::to_string(lineNumber));
                vertices.push_back(make_double3(x, y, z));
            } else if (startsWith(line, "f ")) {
                std::istringstream ss(line.substr(2));
                std::vector<int> corner;
                std::string token;
                const int nv = (int)vertices.size();
                while (ss >> token) {
                    const int id = convertOBJIndexToZeroBased(parseOBJVertexIndex(token), nv);
                    if (id < 0 || id >= nv)
                        throw std::runtime_error("Face index out of range at line " + std::to_string(lineNumber));
                    corner.push_back(id);
                }
                if (corner.size() < 3)
                    throw std::runtime_error("Face has fewer than 3 vertices at line " + std::to_string(lineNumber));
                for (size_t k = 1; k + 1 < corner.size(); ++k)
                    faces.push_back(make_int3(corner[0], corner[k], corner[k + 1]));
            }
        }
    } catch (const std::exception& e) {
        std::cerr << "[OBJLoader] Error while reading " << path << " at line " << lineNumber << ": " << e.what()
                  << std::endl;
        vertices.clear();
        faces.clear();
        return false;
    }
    if (verbose) {
        std::cout << "[OBJLoader] Loaded OBJ: " << path << std::endl;
        std::cout << "  Num vertices = " << vertices.size() << std::endl;
        std::cout << "  Num faces    = " << faces.size() << std::endl;
    }
    return true;
}

}  // namespace OBJLoader
