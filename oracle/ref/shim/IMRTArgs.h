// Build shim replacing the reference's boost::program_options argument table
// (IMRTOpt/include/IMRTArgs.h) with a registry the harness fills directly.
#pragma once
#include <any>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>
namespace IMRT {
std::map<std::string, std::any>& harness_args();
template <class T>
const T& getarg(const std::string& key) {
    auto it = harness_args().find(key);
    if (it == harness_args().end()) {
        std::fprintf(stderr, "harness: missing argument %s\n", key.c_str());
        std::abort();
    }
    return *std::any_cast<T>(&it->second);
}
}
#define VECT2ARR(a, v) a[0] = v.x; a[1] = v.y;
#define VECT3ARR(a, v) a[0] = v.x; a[1] = v.y; a[2] = v.z;
#define ARR2VECT(v, a) v.x = a[0]; v.y = a[1];
#define ARR3VECT(v, a) v.x = a[0]; v.y = a[1]; v.z = a[2];
#define FORMAT_3VEC(v) "("<<v.x<<", "<<v.y<<", "<<v.z<<")"
#define FORMAT_2VEC(v) "("<<v.x<<", "<<v.y<<")"
