// Value types of the LSSolver call surface, symmetric 3x3 matrix (inertia
// tensors) with the names of the reference's myMat.h.
#pragma once
#include "myVec.h"

struct symMatrix {
    double xx, yy, zz, xy, xz, yz;
};

FUNDEM_HD inline symMatrix make_symMatrix(double xx, double yy, double zz, double xy, double xz, double yz)
{
    return symMatrix{xx, yy, zz, xy, xz, yz};
}

FUNDEM_HD inline double3 operator*(const symMatrix& m, const double3 v)
{
    return make_double3(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
                        m.xz * v.x + m.yz * v.y + m.zz * v.z);
}
