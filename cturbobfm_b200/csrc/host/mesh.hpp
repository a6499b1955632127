// Mesh: structured vertex-centred grid and its dual-grid metrics, computed on
// the host in FP64 with the reference's formulas and operation order
// (src/mesh.cpp:11-677, src/input.cpp:14-82, src/math_utils.cpp:173-234,
// 395-463). Compiled with -ffp-contract=off so every metric is bit-identical
// to the reference's.
#pragma once

#include <array>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "config.hpp"

namespace ctbfm {

struct Vec3 {
    double x = 0, y = 0, z = 0;
    Vec3() = default;
    Vec3(double a, double b, double c) : x(a), y(b), z(c) {}
    Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
    Vec3 operator/(double s) const { return {x / s, y / s, z / s}; }
    Vec3 operator-() const { return {-x, -y, -z}; }
    double dot(const Vec3& o) const { return x * o.x + y * o.y + z * o.z; }
    double magnitude() const { return std::sqrt(x * x + y * y + z * z); }
    Vec3 cross(const Vec3& o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
};

class Mesh {
public:
    Mesh(const Config& config);
    // A grid given in memory: ni*nj*nk coordinates and further columns
    // (blockage, blade normals, ...) with node (i, j, k) at (i*nj + j)*nk + k,
    // the grid file's row order. The arrays are copied.
    Mesh(const Config& config, long ni, long nj, long nk, const double* x, const double* y, const double* z,
         const std::vector<std::pair<std::string, const double*>>& fields);

    long ni() const { return ni_; }
    long nj() const { return nj_; }
    long nk() const { return nk_; }
    long nodes() const { return ni_ * nj_ * nk_; }
    int dimensions() const { return ndim_; }

    long idx(long i, long j, long k) const { return (i * nj_ + j) * nk_ + k; }
    long dualIdx(long i, long j, long k) const { return (i * (nj_ + 1) + j) * (nk_ + 1) + k; }
    // face grids: I (ni+1, nj, nk), J (ni, nj+1, nk), K (ni, nj, nk+1)
    long faceIdx(int dir, long i, long j, long k) const;
    long faceCount(int dir) const;

    const std::vector<Vec3>& vertices() const { return vert_; }
    const std::vector<Vec3>& dualNodes() const { return dual_; }
    const std::vector<Vec3>& surfaces(int dir) const { return surf_[dir]; }
    const std::vector<Vec3>& centers(int dir) const { return ctr_[dir]; }
    const std::vector<double>& volumes() const { return vol_; }
    double wedgeAngle() const { return wedge_; }

    bool hasField(const std::string& name) const { return fields_.count(name) > 0; }
    const std::vector<double>& field(const std::string& name) const;

    // Green-Gauss gradient of the blockage (Mesh::computeInputGradients).
    const std::vector<Vec3>& blockageGradient() const { return gradb_; }

    double radius(long i, long j, long k) const {
        const Vec3& p = vert_[idx(i, j, k)];
        return std::sqrt(p.y * p.y + p.z * p.z);
    }
    double theta(long i, long j, long k) const {
        const Vec3& p = vert_[idx(i, j, k)];
        return std::atan2(p.z, p.y);
    }

    // Mesh::checkPeriodicity (src/mesh.cpp:584-619); throws on mismatch.
    void checkPeriodicity(double translation, double angleRad) const;

private:
    void readGrid(const std::string& path);
    void build(const Config& config, const std::string& source);
    void dual2d(bool axisymmetric);
    void dual3d();
    void interfaces();
    void finiteVolumes();
    void blockageGradientGreenGauss();

    long ni_ = 0, nj_ = 0, nk_ = 0;
    int ndim_ = 0;
    Topology topo_;
    std::vector<Vec3> vert_, dual_;
    std::array<std::vector<Vec3>, 3> surf_, ctr_;
    std::vector<double> vol_;
    std::vector<Vec3> gradb_;
    double wedge_ = 0.0;
    std::map<std::string, std::vector<double>> fields_;
};

}  // namespace ctbfm
