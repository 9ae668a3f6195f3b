// Build-time stand-in for the reference's generated OpenCL source map
// (produced by libs/gpu/libgpu/make_source_map.cpp in the reference build).
// The oracle build only calls the reference's CPU functions, so the map of
// embedded kernel sources is empty.
#pragma once
#include <string>
#include <unordered_map>
struct KernelSource {
    const char *kernel;
    size_t length;
};
static const std::unordered_map<std::string, KernelSource> HeadersMap = {};
