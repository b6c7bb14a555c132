// Reads a mesh with include/BAEMM_Meshes.hpp and prints what it read, so the
// tests can compare the C++ readers with the Python ones.
//   mesh_reader txt|stl <path>
#include <cstdio>
#include <string>

#include "BAEMM_Meshes.hpp"

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    std::vector<double> coords;
    std::vector<int64_t> simplices;
    const std::string kind = argv[1];
    const bool ok = kind == "stl" ? BAEMM::ReadMeshFromSTL(argv[2], coords, simplices)
                                  : BAEMM::ReadMeshFromFile(argv[2], coords, simplices);
    if (!ok) return 1;
    std::printf("%zu %zu\n", coords.size() / 3, simplices.size() / 3);
    for (size_t i = 0; i < coords.size(); i += 3) std::printf("%.17g %.17g %.17g\n", coords[i], coords[i + 1], coords[i + 2]);
    for (size_t i = 0; i < simplices.size(); i += 3)
        std::printf("%lld %lld %lld\n", (long long)simplices[i], (long long)simplices[i + 1], (long long)simplices[i + 2]);
    return 0;
}
