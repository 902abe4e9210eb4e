// Minimal stand-ins for the AMReX types and macros that the reference's
// header-only math (Source/interpolants.H, Source/mpm_kernels.H,
// Source/constitutive_models.H, the sampling part of Source/mpm_eb.H) names.
// Written for the oracle's reference pin only; it is not AMReX.
#ifndef EXG_REFPIN_AMREX_SHIM_H_
#define EXG_REFPIN_AMREX_SHIM_H_
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#define AMREX_SPACEDIM 3
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_DEVICE
#define AMREX_GPU_CONSTANT
#define AMREX_FORCE_INLINE inline
#define AMREX_D_DECL(a, b, c) a, b, c

namespace amrex {
using Real = double;
inline void Abort(const std::string &msg) { throw std::runtime_error(msg); }
struct IntVect {
    int v[3] = {0, 0, 0};
    IntVect() = default;
    IntVect(int a, int b, int c) { v[0] = a; v[1] = b; v[2] = c; }
    int &operator[](int i) { return v[i]; }
    int operator[](int i) const { return v[i]; }
};
template <class T, int N>
struct GpuArray {
    T arr[N];
    T &operator[](int i) { return arr[i]; }
    const T &operator[](int i) const { return arr[i]; }
};
struct Dim3 { int x, y, z; };
// Array4: a strided view with inclusive index bounds [lo, hi].
template <class T>
struct Array4 {
    T *p = nullptr;
    Dim3 lo{0, 0, 0}, hi{0, 0, 0};
    long nx() const { return hi.x - lo.x + 1; }
    long ny() const { return hi.y - lo.y + 1; }
    long nz() const { return hi.z - lo.z + 1; }
    T &operator()(int i, int j, int k, int n = 0) const {
        return p[(((long)n * nz() + (k - lo.z)) * ny() + (j - lo.y)) * nx() + (i - lo.x)];
    }
    T &operator()(IntVect iv, int n = 0) const { return (*this)(iv[0], iv[1], iv[2], n); }
};
template <class T> Dim3 lbound(const Array4<T> &a) { return a.lo; }
template <class T> Dim3 ubound(const Array4<T> &a) { return a.hi; }
template <class T> T max(T a, T b) { return a > b ? a : b; }
template <class T> T min(T a, T b) { return a < b ? a : b; }
template <class T> T Clamp(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }
namespace Math {
inline double floor(double x) { return std::floor(x); }
inline double abs(double x) { return std::fabs(x); }
}
}  // namespace amrex
#endif
