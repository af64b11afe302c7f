// VTK XML unstructured-grid files (.vtu) for the frames LSSolver::solve
// writes: points in single precision, optional cells, per-point arrays, and
// the frame's time and step as field data.  Arrays are stored inline in the
// "binary" encoding of the VTK XML format: base64 (RFC 4648) of a 64-bit
// little-endian byte count followed by the raw little-endian values
// (header_type UInt64), which ParaView reads directly.
#pragma once
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace fundem_vtu
{

// base64 of one inline binary block: the 64-bit byte count, then the bytes
inline void base64_block(std::ostream& out, const void* data, size_t nbytes)
{
    static const char table[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::vector<uint8_t> buf(8 + nbytes);
    const uint64_t count = nbytes;
    std::memcpy(buf.data(), &count, 8);
    if (nbytes) std::memcpy(buf.data() + 8, data, nbytes);
    std::string s;
    s.reserve((buf.size() + 2) / 3 * 4);
    for (size_t i = 0; i < buf.size(); i += 3) {
        const size_t left = buf.size() - i;
        const uint32_t w = (uint32_t(buf[i]) << 16) | (left > 1 ? uint32_t(buf[i + 1]) << 8 : 0u) |
                           (left > 2 ? uint32_t(buf[i + 2]) : 0u);
        s += table[(w >> 18) & 63];
        s += table[(w >> 12) & 63];
        s += left > 1 ? table[(w >> 6) & 63] : '=';
        s += left > 2 ? table[w & 63] : '=';
    }
    out << s;
}

// one named per-point array
struct Array {
    std::string name;
    std::string type;  // Float32, Int32 or UInt8
    int components = 1;
    std::vector<uint8_t> bytes;
};

inline const char* vtk_type(float) { return "Float32"; }
inline const char* vtk_type(int32_t) { return "Int32"; }
inline const char* vtk_type(uint8_t) { return "UInt8"; }

template <typename T>
inline Array array(const std::string& name, int components, const std::vector<T>& v)
{
    Array a;
    a.name = name;
    a.type = vtk_type(T());
    a.components = components;
    a.bytes.resize(v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(a.bytes.data(), v.data(), a.bytes.size());
    return a;
}

// Writes one piece: points (xyz per point), cells from connectivity, offsets
// and VTK cell types (all three empty for a point cloud), and point arrays.
// Returns false when the file cannot be written.
inline bool write(const std::string& file, double time, long long step, const std::vector<float>& points,
                  const std::vector<int32_t>& connectivity, const std::vector<int32_t>& offsets,
                  const std::vector<uint8_t>& types, const std::vector<Array>& point_data)
{
    std::ofstream out(file);
    if (!out) return false;
    const size_t n_points = points.size() / 3, n_cells = types.size();
    out << "<?xml version=\"1.0\"?>\n"
        << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
        << "<UnstructuredGrid>\n<FieldData>\n"
        << "<DataArray type=\"Float32\" Name=\"TIME\" NumberOfTuples=\"1\" format=\"ascii\">" << float(time)
        << "</DataArray>\n"
        << "<DataArray type=\"Int32\" Name=\"STEP\" NumberOfTuples=\"1\" format=\"ascii\">" << int32_t(step)
        << "</DataArray>\n</FieldData>\n"
        << "<Piece NumberOfPoints=\"" << n_points << "\" NumberOfCells=\"" << n_cells << "\">\n"
        << "<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">\n";
    base64_block(out, points.data(), points.size() * sizeof(float));
    out << "\n</DataArray>\n</Points>\n<Cells>\n";
    if (n_cells == 0) {
        out << "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\"></DataArray>\n"
            << "<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\"></DataArray>\n"
            << "<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\"></DataArray>\n";
    } else {
        out << "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">\n";
        base64_block(out, connectivity.data(), connectivity.size() * sizeof(int32_t));
        out << "\n</DataArray>\n<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">\n";
        base64_block(out, offsets.data(), offsets.size() * sizeof(int32_t));
        out << "\n</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">\n";
        base64_block(out, types.data(), types.size());
        out << "\n</DataArray>\n";
    }
    out << "</Cells>\n<PointData>\n";
    for (const Array& a : point_data) {
        out << "<DataArray type=\"" << a.type << "\" Name=\"" << a.name << "\"";
        if (a.components > 1) out << " NumberOfComponents=\"" << a.components << "\"";
        out << " format=\"binary\">\n";
        base64_block(out, a.bytes.data(), a.bytes.size());
        out << "\n</DataArray>\n";
    }
    out << "</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
    return bool(out);
}

}  // namespace fundem_vtu
