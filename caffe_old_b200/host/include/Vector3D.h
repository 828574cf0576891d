// Minimal 3-vector of the host layer (the reference's Vector3D / Point3D, src/Math/Vector3D.h),
// with std::stov parsing "(x,y,z)" strings as the reference's case files write them.
#pragma once
#include <string>

class Vector3D {
public:
    double x = 0., y = 0., z = 0.;
    Vector3D() = default;
    Vector3D(double a, double b, double c) : x(a), y(b), z(c) {}
    double& operator()(int i) { return i == 0 ? x : (i == 1 ? y : z); }
    double operator()(int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    Vector3D operator+(const Vector3D& o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vector3D operator-(const Vector3D& o) const { return {x - o.x, y - o.y, z - o.z}; }
    Vector3D operator*(double s) const { return {x * s, y * s, z * s}; }
};
inline Vector3D operator*(double s, const Vector3D& v) { return v * s; }
typedef Vector3D Point3D;

namespace std {
// "(x,y,z)" -> Vector3D (Vector3D.cpp's stov); throws const char* on malformed input
Vector3D stov(const std::string& s);
}
