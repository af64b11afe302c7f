// Exercises the file helpers of myFileEdit.h in the directory given as the
// first argument: prints each extension test on a list of names, then each
// remove function's count and the entries left after it.  Built against this
// library's header and against the reference's, the outputs must agree.
#include <algorithm>
#include <cstdio>
#include <filesystem>
#include <string>
#include <vector>

#include "CUDAKernelFunction/myUtility/myFileEdit.h"

static void listing(const std::string& dir)
{
    std::vector<std::string> names;
    for (const auto& e : std::filesystem::directory_iterator(dir)) names.push_back(e.path().filename().string());
    std::sort(names.begin(), names.end());
    for (const std::string& n : names) std::printf("  %s\n", n.c_str());
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    const char* names[] = {"a.vtu", "a.VTU", "a.vtu.bak", ".vtu", "vtu", "b.vtm", "c.vti", "d.obj", "e.dat", "f."};
    for (const char* n : names)
        std::printf("%s %d %d %d %d %d\n", n, (int)hasVtuExt(n), (int)hasVtmExt(n), (int)hasVtiExt(n),
                    (int)hasObjExt(n), (int)hasDatExt(n));
    std::printf("missing %d\n", removeVtuFiles(dir + "/no_such_dir"));
    std::printf("vtu %d\n", removeVtuFiles(dir));
    listing(dir);
    std::printf("vtm %d\n", removeVtmFiles(dir));
    std::printf("vti %d\n", removeVtiFiles(dir));
    std::printf("obj %d\n", removeObjFiles(dir));
    std::printf("dat %d\n", removeDatFiles(dir));
    listing(dir);
    const std::string made = dir + "/made";
    const int first = MKDIR(made.c_str());
    const int again = MKDIR(made.c_str());
    std::printf("mkdir %d %d\n", first, again);
    return 0;
}
