// Value types of the LSSolver call surface, vector part.
//
// Apps written against FunDEM use CUDA's double3 / int3 with free functions
// and operators of these names (reference: kernel/CUDAKernelFunction/
// myUtility/myVec.h).  They are reproduced here under the same names so that
// such apps compile unchanged against this library; the arithmetic is plain
// and is not used on the library's own kernels.
#pragma once
#include <cmath>
#include <vector_functions.h>
#include <vector_types.h>

#if defined(__CUDACC__)
#define FUNDEM_HD __host__ __device__
#else
#define FUNDEM_HD
#endif

FUNDEM_HD inline double pi() { return 3.14159265358979323846; }
// the reference's zero test: |x| <= 1e-20
FUNDEM_HD inline bool isZero(const double x) { return fabs(x) <= 1.0e-20; }

FUNDEM_HD inline double3 operator+(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
FUNDEM_HD inline double3 operator-(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
FUNDEM_HD inline double3 operator-(double3 a) { return make_double3(-a.x, -a.y, -a.z); }
FUNDEM_HD inline double3 operator*(double3 a, double s) { return make_double3(a.x * s, a.y * s, a.z * s); }
FUNDEM_HD inline double3 operator*(double s, double3 a) { return make_double3(s * a.x, s * a.y, s * a.z); }
// division by a scalar multiplies by its reciprocal, as the reference's value type does (myVec.h:55-59)
FUNDEM_HD inline double3 operator/(double3 a, double s)
{
    const double inv = 1.0 / s;
    return make_double3(a.x * inv, a.y * inv, a.z * inv);
}
FUNDEM_HD inline double3& operator+=(double3& a, double3 b) { a = a + b; return a; }
FUNDEM_HD inline double3& operator-=(double3& a, double3 b) { a = a - b; return a; }
FUNDEM_HD inline double3& operator*=(double3& a, double s) { a = a * s; return a; }
FUNDEM_HD inline double3& operator/=(double3& a, double s) { a = a / s; return a; }

FUNDEM_HD inline double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
FUNDEM_HD inline double3 cross(double3 a, double3 b)
{
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
FUNDEM_HD inline double lengthSquared(double3 v) { return dot(v, v); }
FUNDEM_HD inline double length(double3 v) { return sqrt(dot(v, v)); }
// unit vector; the zero vector stays zero
FUNDEM_HD inline double3 normalize(double3 v)
{
    const double l2 = dot(v, v);
    if (isZero(l2)) return make_double3(0.0, 0.0, 0.0);
    return v * (1.0 / sqrt(l2));
}

// x-fastest linear index of cell (x, y, z) in a grid of the given size
FUNDEM_HD inline int linearIndex3D(const int3 ijk, const int3 dims)
{
    return ijk.z * dims.y * dims.x + ijk.y * dims.x + ijk.x;
}
