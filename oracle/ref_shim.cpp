// C entry points over the reference's own geometry code (src/Math/Geometry.cpp, Sphere.cpp,
// Vector3D.cpp, Tensor3D.cpp) and its Array3D container (src/DataStructures/Array3D.h/.tpp),
// compiled where they lie by `make -C oracle ref` into oracle/_ref/libref_geometry.so.  Test
// infrastructure only: it pins the oracle's mesh-metric and immersed-boundary geometry, and
// its cell storage order, against the reference's code.
#include "Array3D.h"
#include "Geometry.h"
#include "Sphere.h"
#include "Tensor3D.h"

namespace {
void load(const double* p, int n, Point3D* out) {
    for (int q = 0; q < n; ++q) out[q] = Point3D(p[3 * q], p[3 * q + 1], p[3 * q + 2]);
}
}  // namespace

extern "C" {
double ref_hex_volume(const double* p24) {
    Point3D p[8];
    load(p24, 8, p);
    return Geometry::computeHexahedronVolume(p);
}
void ref_hex_centroid(const double* p24, double* out) {
    Point3D p[8];
    load(p24, 8, p);
    Point3D c = Geometry::computeHexahedronCentroid(p);
    out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
double ref_quad_area(const double* p12) {
    Point3D p[4];
    load(p12, 4, p);
    return Geometry::computeQuadrilateralArea(p);
}
void ref_quad_centroid(const double* p12, double* out) {
    Point3D p[4];
    load(p12, 4, p);
    Point3D c = Geometry::computeQuadrilateralCentroid(p);
    out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
int ref_inside_hex(const double* pt, const double* p24) {
    Point3D p[8];
    load(p24, 8, p);
    return Geometry::isInsideHexahedron(Point3D(pt[0], pt[1], pt[2]), p) ? 1 : 0;
}
void ref_nearest_intersect(double radius, const double* center, const double* pt, double* out) {
    Sphere s(radius, Point3D(center[0], center[1], center[2]));
    Point3D r = s.nearestIntersect(Point3D(pt[0], pt[1], pt[2]));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
// face vector (unit normal times area) of a quadrilateral, as the mesh set-up composes it
// from the reference's Vector3D and Geometry routines (HexaFvmMesh.cpp:722-727)
void ref_face_vector(const double* p12, double* out) {
    Point3D p[4];
    load(p12, 4, p);
    Vector3D n = cross(p[1] - p[0], p[2] - p[0]).unitVector() * Geometry::computeQuadrilateralArea(p);
    out[0] = n.x; out[1] = n.y; out[2] = n.z;
}
// diffusion metric D_f = |S|^2 / (S . r) and non-orthogonal vector c_f = S - r |S|^2 / (S . r)
// of one cell face, in the reference's Vector3D arithmetic (HexaFvmMesh.cpp:872-884): out =
// (D, c.x, c.y, c.z)
void ref_d_and_c(const double* s3, const double* r3, double* out) {
    Vector3D s(s3[0], s3[1], s3[2]), r(r3[0], r3[1], r3[2]);
    double d = dot(s, s) / dot(s, r);
    Vector3D c = s - r * dot(s, s) / dot(s, r);
    out[0] = d; out[1] = c.x; out[2] = c.y; out[3] = c.z;
}
// divergence-theorem velocity gradient of one cell from its six face velocities and outward
// face vectors (E W N S T B), in the reference's Vector3D / Tensor3D arithmetic
// (FvVectorScheme.cpp:64-69): out = 9 entries, row-major
void ref_grad_tensor(const double* uf18, const double* s18, double volume, double* out) {
    Vector3D u[6], s[6];
    for (int f = 0; f < 6; ++f) {
        u[f] = Vector3D(uf18[3 * f], uf18[3 * f + 1], uf18[3 * f + 2]);
        s[f] = Vector3D(s18[3 * f], s18[3 * f + 1], s18[3 * f + 2]);
    }
    Tensor3D g = (tensor(u[0], s[0]) + tensor(u[1], s[1]) + tensor(u[2], s[2]) + tensor(u[3], s[3]) + tensor(u[4], s[4]) +
                  tensor(u[5], s[5])) / volume;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) out[3 * r + c] = g(r, c);
}
// offset of element (i, j, k) in an Array3D of sizeI x sizeJ x sizeK, or -1 where the
// reference's bounds-checked operator() throws
long ref_array3d_offset(int sizeI, int sizeJ, int sizeK, int i, int j, int k) {
    Array3D<double> a(sizeI, sizeJ, sizeK);
    try {
        return (long)(&a(i, j, k) - a.data());
    } catch (const char*) {
        return -1;
    }
}
// image point of a ghost-cell centre x: 2 BP - x with BP the sphere's nearest intersection,
// in the reference's Vector3D arithmetic (IbPiso.cpp:137-138)
void ref_image_point(double radius, const double* center, const double* x, double* out) {
    Sphere s(radius, Point3D(center[0], center[1], center[2]));
    Point3D xg(x[0], x[1], x[2]);
    Point3D bp = s.nearestIntersect(xg);
    Point3D ip = 2. * bp - xg;
    out[0] = ip.x; out[1] = ip.y; out[2] = ip.z;
}
int ref_sphere_is_inside(double radius, const double* center, const double* pt) {
    Sphere s(radius, Point3D(center[0], center[1], center[2]));
    return s.isInside(Point3D(pt[0], pt[1], pt[2])) ? 1 : 0;
}
}
