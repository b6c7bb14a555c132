// BAEMM_Meshes.hpp -- header-only mesh readers for the B200 BAEMM library.
//
// BAEMM::ReadMeshFromFile  the reference's text format (ReadMeshFromFile.hpp:3-102):
//                          "dom_dim d amb_dim a vertex_count n simplex_count m",
//                          then n rows of a coordinates and m rows of d+1
//                          0-based vertex indices.
// BAEMM::ReadMeshFromSTL   STL files (ReadMeshFromSTL.hpp:5-44), ASCII or binary.
//
// Both fill row-major std::vectors (coords: vertex_count x 3 doubles,
// simplices: simplex_count x 3 int64) instead of the reference's Tensor2, and
// return false (after printing the reason to std::cerr) where the reference
// prints an error and returns false.  The result feeds the Helmholtz_CUDA
// constructor directly (coords.data(), simplices.data()).
//
// The reference reads STL through the stl_reader library (an unvendored
// submodule).  Its published behaviour, restated here: a binary file is an
// 80-byte header, a uint32 triangle count and 50 bytes per triangle (normal,
// three vertices as float32, a uint16 attribute); an ASCII file is a sequence of
// "solid ... facet normal ... outer loop vertex x y z (x3) endloop endfacet ...
// endsolid" blocks (several solids allowed).  Vertices with bit-identical
// float coordinates are merged; the unique vertices are numbered in
// lexicographic (x, y, z) order and the triangles keep their file order.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

namespace BAEMM
{

inline bool ReadMeshFromFile(const std::string &file, std::vector<double> &coords, std::vector<int64_t> &simplices)
{
    const std::string tag = "ReadMeshFromFile";
    std::ifstream s(file);
    if (!s.good())
    {
        std::cerr << tag << ": File " << file << " could not be opened.\n";
        return false;
    }
    const char *keys[4] = {"dom_dim", "amb_dim", "vertex_count", "simplex_count"};
    int64_t v[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k)
    {
        std::string str;
        s >> str;
        if (str != keys[k] || !(s >> v[k]) || v[k] < 0)
        {
            std::cerr << tag << ": Invalid file (expected " << keys[k] << "). Aborting.\n";
            return false;
        }
    }
    const int64_t dom_dim = v[0], amb_dim = v[1], n = v[2], m = v[3];
    if (amb_dim != 3 || dom_dim != 2)
    {
        std::cerr << tag << ": only triangle meshes in 3D (dom_dim 2, amb_dim 3) are supported.\n";
        return false;
    }
    coords.resize((size_t)(n * amb_dim));
    simplices.resize((size_t)(m * (dom_dim + 1)));
    for (auto &x : coords)
        if (!(s >> x))
        {
            std::cerr << tag << ": File " << file << " is truncated.\n";
            return false;
        }
    for (auto &t : simplices)
        if (!(s >> t) || t < 0 || t >= n)
        {
            std::cerr << tag << ": File " << file << " is truncated or has an invalid vertex index.\n";
            return false;
        }
    return true;
}

namespace detail
{
// Merge bit-identical vertices; unique vertices in lexicographic order.
inline void stl_index(const std::vector<float> &raw, std::vector<double> &coords, std::vector<int64_t> &simplices)
{
    const size_t nraw = raw.size() / 3;
    std::vector<size_t> order(nraw);
    for (size_t i = 0; i < nraw; ++i) order[i] = i;
    auto less = [&](size_t a, size_t b) {
        for (int d = 0; d < 3; ++d)
        {
            const float x = raw[3 * a + d], y = raw[3 * b + d];
            if (x < y) return true;
            if (y < x) return false;
        }
        return false;
    };
    std::sort(order.begin(), order.end(), less);
    std::vector<int64_t> id(nraw, 0);
    coords.clear();
    int64_t next = -1;
    for (size_t k = 0; k < nraw; ++k)
    {
        const size_t i = order[k];
        if (k == 0 || less(order[k - 1], i))
        {
            ++next;
            for (int d = 0; d < 3; ++d) coords.push_back((double)raw[3 * i + d]);
        }
        id[i] = next;
    }
    simplices.resize(nraw);
    for (size_t i = 0; i < nraw; ++i) simplices[i] = id[i];   // raw vertex i is corner i % 3 of triangle i / 3
}
} // namespace detail

inline bool ReadMeshFromSTL(const std::string &file, std::vector<double> &coords, std::vector<int64_t> &simplices)
{
    const std::string tag = "ReadMeshFromSTL";
    std::ifstream s(file, std::ios::binary);
    if (!s.good())
    {
        std::cerr << tag << ": File " << file << " could not be opened.\n";
        return false;
    }
    const std::vector<char> bytes((std::istreambuf_iterator<char>(s)), std::istreambuf_iterator<char>());
    std::vector<float> raw;   // 9 floats per triangle
    bool binary = false;
    if (bytes.size() >= 84)
    {
        uint32_t count = 0;
        std::memcpy(&count, bytes.data() + 80, 4);
        binary = (uint64_t)bytes.size() == 84ull + 50ull * count;
        if (binary)
        {
            raw.resize((size_t)count * 9);
            for (uint32_t t = 0; t < count; ++t)
                std::memcpy(&raw[(size_t)t * 9], bytes.data() + 84 + 50 * (size_t)t + 12, 36);
        }
    }
    if (!binary)
    {
        std::string text(bytes.begin(), bytes.end());
        std::istringstream in(text);
        std::string tok;
        if (!(in >> tok) || tok != "solid")
        {
            std::cerr << tag << ": " << file << " is neither binary STL nor ASCII STL.\n";
            return false;
        }
        while (in >> tok)
        {
            if (tok != "vertex") continue;
            float x, y, z;
            if (!(in >> x >> y >> z))
            {
                std::cerr << tag << ": " << file << ": malformed vertex.\n";
                return false;
            }
            raw.push_back(x);
            raw.push_back(y);
            raw.push_back(z);
        }
        if (raw.size() % 9 != 0)
        {
            std::cerr << tag << ": " << file << ": vertex count is not a multiple of 3.\n";
            return false;
        }
    }
    detail::stl_index(raw, coords, simplices);
    return true;
}

} // namespace BAEMM
