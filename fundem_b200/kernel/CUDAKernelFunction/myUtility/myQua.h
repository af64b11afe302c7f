// Value types of the LSSolver call surface, orientation part: the quaternion
// (scalar first) with the names of the reference's myQua.h.
#pragma once
#include "myVec.h"

struct quaternion {
    double q0, q1, q2, q3;
};

FUNDEM_HD inline quaternion make_quaternion(double q0, double q1, double q2, double q3)
{
    return quaternion{q0, q1, q2, q3};
}

// unit quaternion; a zero quaternion is returned unchanged
FUNDEM_HD inline quaternion normalize(quaternion q)
{
    const double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
    if (isZero(l2)) return q;
    const double s = 1.0 / sqrt(l2);
    return quaternion{q.q0 * s, q.q1 * s, q.q2 * s, q.q3 * s};
}

// v rotated by the unit quaternion q (body frame -> world frame)
FUNDEM_HD inline double3 rotateVectorByQuaternion(const quaternion q, const double3 v)
{
    const double3 u = make_double3(q.q1, q.q2, q.q3);
    const double3 t = 2.0 * cross(u, v);
    return v + q.q0 * t + cross(u, t);
}

// v rotated by the inverse of q (world frame -> body frame)
FUNDEM_HD inline double3 reverseRotateVectorByQuaternion(const double3 v, const quaternion q)
{
    return rotateVectorByQuaternion(quaternion{q.q0, -q.q1, -q.q2, -q.q3}, v);
}
