// Counter-based random numbers shared by the host initialisers and the device kernels.
// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014) applied to a key built from (seed, stream, a, b); the uniform variate keeps the top
// 53 bits.  Identical on host and device, so every initial state and parameter table can be
// regenerated anywhere from its seed.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define OPGPU_HD __host__ __device__ __forceinline__
#else
#define OPGPU_HD inline
#endif

namespace opgpu {

enum : uint64_t {
    kStreamPosition = 1,   // Voronoi seed / nucleus positions (b = axis)
    kStreamSigma    = 2,   // per-grain-pair interface energy (a < b)
    kStreamDrivingForce = 3,
    kStreamMobility = 4,
    kStreamOrientation = 5,
};

OPGPU_HD uint64_t splitmix64(uint64_t x)
{
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

OPGPU_HD uint64_t key64(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b)
{
    uint64_t h = splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ull));
    h = splitmix64(h ^ a);
    h = splitmix64(h ^ (b * 0x8CB92BA72F3D8DD7ull));
    return h;
}

OPGPU_HD double uniform01(uint64_t seed, uint64_t stream, uint64_t a, uint64_t b)
{
    return (double)(key64(seed, stream, a, b) >> 11) * 0x1.0p-53;
}

}  // namespace opgpu
