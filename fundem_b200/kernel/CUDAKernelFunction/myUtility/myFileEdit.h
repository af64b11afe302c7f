// File helpers of the reference's kernel/CUDAKernelFunction/myUtility/
// myFileEdit.h, which LSParticle.h includes, so apps that include LSSolver.h
// see them: MKDIR(path), the extension tests hasVtuExt / hasVtmExt /
// hasVtiExt / hasObjExt / hasDatExt, and removeVtuFiles / removeVtmFiles /
// removeVtiFiles / removeObjFiles / removeDatFiles.
//
// The tests look at the text after the last '.' of a name, exactly (".vtu",
// not ".VTU").  A remove function deletes the entries of `dir` (not of its
// subdirectories) with that extension, skipping directories themselves but
// not links to them, and returns how many it deleted; 0 when `dir` cannot be
// read.  POSIX only.
#pragma once
#include <cstdio>
#include <cstring>
#include <string>
#include <system_error>
#include <filesystem>

#include <sys/stat.h>

#define MKDIR(path) mkdir(path, 0755)

namespace fundem_file_detail
{
inline bool hasExt(const char* fname, const char* ext)
{
    const char* dot = std::strrchr(fname, '.');
    return dot != nullptr && std::strcmp(dot, ext) == 0;
}

inline int removeWithExt(const std::string& dir, const char* ext)
{
    namespace fs = std::filesystem;
    std::error_code ec;
    fs::directory_iterator it(dir, ec), end;
    if (ec) return 0;
    int removed = 0;
    for (; it != end; it.increment(ec)) {
        if (ec) break;
        std::error_code sec;
        // the entry itself, links not followed
        if (it->symlink_status(sec).type() == fs::file_type::directory) continue;
        const std::string name = it->path().filename().string();
        if (!hasExt(name.c_str(), ext)) continue;
        if (std::remove((dir + "/" + name).c_str()) == 0) ++removed;
    }
    return removed;
}
}  // namespace fundem_file_detail

static inline bool hasVtuExt(const char* fname) { return fundem_file_detail::hasExt(fname, ".vtu"); }
static inline bool hasVtmExt(const char* fname) { return fundem_file_detail::hasExt(fname, ".vtm"); }
static inline bool hasVtiExt(const char* fname) { return fundem_file_detail::hasExt(fname, ".vti"); }
static inline bool hasObjExt(const char* fname) { return fundem_file_detail::hasExt(fname, ".obj"); }
static inline bool hasDatExt(const char* fname) { return fundem_file_detail::hasExt(fname, ".dat"); }

static inline int removeVtuFiles(const std::string& dir) { return fundem_file_detail::removeWithExt(dir, ".vtu"); }
static inline int removeVtmFiles(const std::string& dir) { return fundem_file_detail::removeWithExt(dir, ".vtm"); }
static inline int removeVtiFiles(const std::string& dir) { return fundem_file_detail::removeWithExt(dir, ".vti"); }
static inline int removeObjFiles(const std::string& dir) { return fundem_file_detail::removeWithExt(dir, ".obj"); }
static inline int removeDatFiles(const std::string& dir) { return fundem_file_detail::removeWithExt(dir, ".dat"); }
