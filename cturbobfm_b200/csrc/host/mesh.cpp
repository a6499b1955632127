// Mesh: see mesh.hpp.
#include "mesh.hpp"

#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ctbfm {

Mesh::Mesh(const Config& config) : topo_(config.getTopology()) {
    std::string path = config.gridFilePath();
    if (!path.empty() && path[0] != '/') path = config.directory() + "/" + path;
    readGrid(path);
    build(config, path);
}

Mesh::Mesh(const Config& config, long ni, long nj, long nk, const double* x, const double* y, const double* z,
           const std::vector<std::pair<std::string, const double*>>& fields)
    : ni_(ni), nj_(nj), nk_(nk), topo_(config.getTopology()) {
    if (ni < 1 || nj < 1 || nk < 1) throw ConfigError("the grid needs ni, nj, nk >= 1");
    if (nj > (1L << 40) / ni || nk > (1L << 40) / (ni * nj)) throw ConfigError("the grid is too large");
    if (!x || !y || !z) throw ConfigError("the grid needs x, y and z");
    const long n = ni * nj * nk;
    vert_.resize(n);
    for (long q = 0; q < n; q++) vert_[q] = Vec3(x[q], y[q], z[q]);
    for (const auto& f : fields) {
        if (f.first.empty() || !f.second) throw ConfigError("a grid field needs a name and values");
        if (f.first == "x" || f.first == "y" || f.first == "z" || fields_.count(f.first))
            throw ConfigError("grid field " + f.first + " given twice");
        fields_[f.first].assign(f.second, f.second + n);
    }
    ndim_ = (nj_ == 1 && nk_ == 1) ? 1 : (nk_ == 1 ? 2 : 3);
    build(config, "the grid arrays");
}

// The dual grid and every metric, from the vertices (src/mesh.cpp:11-677).
void Mesh::build(const Config& config, const std::string& source) {
    if (topo_ == Topology::OneD) throw ConfigError("1-D topology is outside this library's scope");
    if ((topo_ == Topology::ThreeD) != (nk_ > 1))
        throw ConfigError("TOPOLOGY does not match the grid's NK");
    if (ni_ < 3 || nj_ < 3 || (topo_ == Topology::ThreeD && nk_ < 3))
        throw ConfigError("the grid needs at least 3 nodes along every swept direction");
    dual_.assign((ni_ + 1) * (nj_ + 1) * (nk_ + 1), Vec3());
    if (topo_ == Topology::ThreeD) dual3d();
    else dual2d(topo_ == Topology::Axisymmetric);
    interfaces();
    finiteVolumes();
    if (config.isBFMActive()) {
        if (!hasField("blockage")) throw ConfigError("blockage not found in: " + source);
        blockageGradientGreenGauss();
    }
}

const std::vector<double>& Mesh::field(const std::string& name) const {
    auto it = fields_.find(name);
    if (it == fields_.end()) throw ConfigError(name + " not found in the grid file");
    return it->second;
}

long Mesh::faceIdx(int dir, long i, long j, long k) const {
    if (dir == 0) return (i * nj_ + j) * nk_ + k;
    if (dir == 1) return (i * (nj_ + 1) + j) * nk_ + k;
    return (i * nj_ + j) * (nk_ + 1) + k;
}

long Mesh::faceCount(int dir) const {
    if (dir == 0) return (ni_ + 1) * nj_ * nk_;
    if (dir == 1) return ni_ * (nj_ + 1) * nk_;
    return ni_ * nj_ * (nk_ + 1);
}

// Input::readCsvFile (src/input.cpp:14-82).
void Mesh::readGrid(const std::string& path) {
    std::ifstream file(path);
    if (!file) throw ConfigError("Error opening coordinates CSV file '" + path + "'!");
    std::string line;
    std::vector<std::string> headers;
    while (std::getline(file, line)) {
        if (line.rfind("NI=", 0) == 0) ni_ = std::stol(line.substr(3));
        else if (line.rfind("NJ=", 0) == 0) nj_ = std::stol(line.substr(3));
        else if (line.rfind("NK=", 0) == 0) nk_ = std::stol(line.substr(3));
        else if (line.rfind("x,y,z", 0) == 0) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            std::istringstream hs(line);
            std::string col;
            while (std::getline(hs, col, ',')) headers.push_back(col);
            break;
        }
    }
    const long n = ni_ * nj_ * nk_;
    if (n <= 0 || headers.size() < 3) throw ConfigError("bad grid header in " + path);
    std::vector<std::vector<double>> cols(headers.size(), std::vector<double>(n));
    long np = 0;
    std::vector<double> vals(headers.size());
    while (np < n && std::getline(file, line)) {
        const char* p = line.c_str();
        size_t nv = 0;
        while (*p && nv < headers.size() + 1) {
            char* end;
            const double v = std::strtod(p, &end);
            if (end == p) break;
            if (nv < vals.size()) vals[nv] = v;
            nv++;
            p = end;
            while (*p == ',' || *p == ' ') p++;
            if (*p == '\r' || *p == '\n') break;
        }
        if (nv != headers.size()) continue;  // incomplete lines are skipped
        for (size_t h = 0; h < headers.size(); h++) cols[h][np] = vals[h];
        np++;
    }
    if (np != n) throw ConfigError("Number of points in the input file is not equal to ni*nj*nk");
    vert_.resize(n);
    for (size_t h = 0; h < headers.size(); h++) {
        if (headers[h] == "x") for (long q = 0; q < n; q++) vert_[q].x = cols[h][q];
        else if (headers[h] == "y") for (long q = 0; q < n; q++) vert_[q].y = cols[h][q];
        else if (headers[h] == "z") for (long q = 0; q < n; q++) vert_[q].z = cols[h][q];
        else fields_[headers[h]] = std::move(cols[h]);
    }
    ndim_ = (nj_ == 1 && nk_ == 1) ? 1 : (nk_ == 1 ? 2 : 3);
}

// Mesh::computeDualGrid2dTopology (src/mesh.cpp:373-435).
void Mesh::dual2d(bool axisymmetric) {
    const long DI = ni_ + 1, DJ = nj_ + 1;
    std::vector<Vec3> nodes(DI * DJ);
    auto N = [&](long i, long j) -> Vec3& { return nodes[i * DJ + j]; };
    auto V = [&](long i, long j) -> const Vec3& { return vert_[idx(i, j, 0)]; };
    for (long i = 1; i < DI - 1; i++)
        for (long j = 1; j < DJ - 1; j++) N(i, j) = (V(i - 1, j - 1) + V(i, j - 1) + V(i, j) + V(i - 1, j)) / 4.0;
    N(0, 0) = V(0, 0);
    N(0, DJ - 1) = V(0, nj_ - 1);
    N(DI - 1, 0) = V(ni_ - 1, 0);
    N(DI - 1, DJ - 1) = V(ni_ - 1, nj_ - 1);
    for (long i = 1; i < DI - 1; i++) {
        N(i, 0) = (V(i - 1, 0) + V(i, 0)) / 2.0;
        N(i, DJ - 1) = (V(i - 1, nj_ - 1) + V(i, nj_ - 1)) / 2.0;
    }
    for (long j = 1; j < DJ - 1; j++) {
        N(0, j) = (V(0, j - 1) + V(0, j)) / 2.0;
        N(DI - 1, j) = (V(ni_ - 1, j - 1) + V(ni_ - 1, j)) / 2.0;
    }
    if (axisymmetric) {
        wedge_ = 1.0 * M_PI / 180.0;  // 1 degree wedge
        for (long i = 0; i < DI; i++)
            for (long j = 0; j < DJ; j++) {
                Vec3& d0 = dual_[dualIdx(i, j, 0)];
                Vec3& d1 = dual_[dualIdx(i, j, 1)];
                d0.x = N(i, j).x;
                d1.x = N(i, j).x;
                d0.y = N(i, j).y * std::cos(-wedge_ / 2.0);
                d1.y = N(i, j).y * std::cos(+wedge_ / 2.0);
                d0.z = N(i, j).y * std::sin(-wedge_ / 2.0);
                d1.z = N(i, j).y * std::sin(+wedge_ / 2.0);
            }
    } else {
        const double thick = 1.0;  // unit thickness
        for (long i = 0; i < DI; i++)
            for (long j = 0; j < DJ; j++) {
                Vec3& d0 = dual_[dualIdx(i, j, 0)];
                Vec3& d1 = dual_[dualIdx(i, j, 1)];
                d0 = Vec3(N(i, j).x, N(i, j).y, -thick / 2.0);
                d1 = Vec3(N(i, j).x, N(i, j).y, +thick / 2.0);
            }
    }
}

// Mesh::computeDualGrid3dTopology (src/mesh.cpp:478-557).
void Mesh::dual3d() {
    const long NI = ni_, NJ = nj_, NK = nk_, DI = NI + 1, DJ = NJ + 1, DK = NK + 1;
    auto D = [&](long i, long j, long k) -> Vec3& { return dual_[dualIdx(i, j, k)]; };
    auto V = [&](long i, long j, long k) -> const Vec3& { return vert_[idx(i, j, k)]; };
    for (long i = 1; i < DI - 1; i++)
        for (long j = 1; j < DJ - 1; j++)
            for (long k = 1; k < DK - 1; k++)
                D(i, j, k) = (V(i - 1, j - 1, k - 1) + V(i, j - 1, k - 1) + V(i - 1, j, k - 1) + V(i - 1, j - 1, k) +
                              V(i, j, k - 1) + V(i, j - 1, k) + V(i - 1, j, k) + V(i, j, k)) / 8.0;
    D(0, 0, 0) = V(0, 0, 0);
    D(DI - 1, 0, 0) = V(NI - 1, 0, 0);
    D(0, DJ - 1, 0) = V(0, NJ - 1, 0);
    D(0, 0, DK - 1) = V(0, 0, NK - 1);
    D(DI - 1, DJ - 1, 0) = V(NI - 1, NJ - 1, 0);
    D(DI - 1, 0, DK - 1) = V(NI - 1, 0, NK - 1);
    D(0, DJ - 1, DK - 1) = V(0, NJ - 1, NK - 1);
    D(DI - 1, DJ - 1, DK - 1) = V(NI - 1, NJ - 1, NK - 1);
    for (long i = 1; i < DI - 1; i++) {
        D(i, 0, 0) = (V(i - 1, 0, 0) + V(i, 0, 0)) / 2.0;
        D(i, DJ - 1, 0) = (V(i - 1, NJ - 1, 0) + V(i, NJ - 1, 0)) / 2.0;
        D(i, 0, DK - 1) = (V(i - 1, 0, NK - 1) + V(i, 0, NK - 1)) / 2.0;
        D(i, DJ - 1, DK - 1) = (V(i - 1, NJ - 1, NK - 1) + V(i, NJ - 1, NK - 1)) / 2.0;
    }
    for (long j = 1; j < DJ - 1; j++) {
        D(0, j, 0) = (V(0, j - 1, 0) + V(0, j, 0)) / 2.0;
        D(DI - 1, j, 0) = (V(NI - 1, j - 1, 0) + V(NI - 1, j, 0)) / 2.0;
        D(0, j, DK - 1) = (V(0, j - 1, NK - 1) + V(0, j, NK - 1)) / 2.0;
        D(DI - 1, j, DK - 1) = (V(NI - 1, j - 1, NK - 1) + V(NI - 1, j, NK - 1)) / 2.0;
    }
    for (long k = 1; k < DK - 1; k++) {
        D(0, 0, k) = (V(0, 0, k - 1) + V(0, 0, k)) / 2.0;
        D(DI - 1, 0, k) = (V(NI - 1, 0, k - 1) + V(NI - 1, 0, k)) / 2.0;
        D(0, DJ - 1, k) = (V(0, NJ - 1, k - 1) + V(0, NJ - 1, k)) / 2.0;
        D(DI - 1, DJ - 1, k) = (V(NI - 1, NJ - 1, k - 1) + V(NI - 1, NJ - 1, k)) / 2.0;
    }
    for (long j = 1; j < DJ - 1; j++)
        for (long k = 1; k < DK - 1; k++) {
            D(0, j, k) = (V(0, j - 1, k - 1) + V(0, j, k - 1) + V(0, j - 1, k) + V(0, j, k)) / 4.0;
            D(DI - 1, j, k) = (V(NI - 1, j - 1, k - 1) + V(NI - 1, j, k - 1) + V(NI - 1, j - 1, k) + V(NI - 1, j, k)) / 4.0;
        }
    for (long i = 1; i < DI - 1; i++)
        for (long k = 1; k < DK - 1; k++) {
            D(i, 0, k) = (V(i - 1, 0, k - 1) + V(i, 0, k - 1) + V(i - 1, 0, k) + V(i, 0, k)) / 4.0;
            D(i, DJ - 1, k) = (V(i - 1, NJ - 1, k - 1) + V(i, NJ - 1, k - 1) + V(i - 1, NJ - 1, k) + V(i, NJ - 1, k)) / 4.0;
        }
    for (long i = 1; i < DI - 1; i++)
        for (long j = 1; j < DJ - 1; j++) {
            D(i, j, 0) = (V(i - 1, j - 1, 0) + V(i, j - 1, 0) + V(i - 1, j, 0) + V(i, j, 0)) / 4.0;
            D(i, j, DK - 1) = (V(i - 1, j - 1, NK - 1) + V(i, j - 1, NK - 1) + V(i - 1, j, NK - 1) + V(i, j, NK - 1)) / 4.0;
        }
}

namespace {
// Mesh::computeSurfaceVectorAndCenter (src/mesh.cpp:165-190): two triangles.
void surfaceAndCenter(const Vec3& p1, const Vec3& p2, const Vec3& p3, const Vec3& p4, Vec3& normal, Vec3& center) {
    const Vec3 a1 = p2 - p1, b1 = p3 - p2, a2 = p3 - p1, b2 = p4 - p3;
    const Vec3 s1 = a1.cross(b1) / 2.0;
    const Vec3 s2 = a2.cross(b2) / 2.0;
    normal = s1 + s2;
    const Vec3 c1 = (p1 + p2 + p3) / 3.0;
    const Vec3 c2 = (p1 + p3 + p4) / 3.0;
    center = (c1 * s1.magnitude() + c2 * s2.magnitude()) / (s1.magnitude() + s2.magnitude());
}
}  // namespace

// Mesh::computeMeshInterfaces (src/mesh.cpp:116-163).
void Mesh::interfaces() {
    const long DI = ni_ + 1, DJ = nj_ + 1, DK = nk_ + 1;
    for (int d = 0; d < 3; d++) {
        surf_[d].assign(faceCount(d), Vec3());
        ctr_[d].assign(faceCount(d), Vec3());
    }
    auto D = [&](long i, long j, long k) -> const Vec3& { return dual_[dualIdx(i, j, k)]; };
    for (long i = 0; i < DI; i++)
        for (long j = 0; j < DJ - 1; j++)
            for (long k = 0; k < DK - 1; k++)
                surfaceAndCenter(D(i, j, k), D(i, j + 1, k), D(i, j + 1, k + 1), D(i, j, k + 1),
                                 surf_[0][faceIdx(0, i, j, k)], ctr_[0][faceIdx(0, i, j, k)]);
    for (long i = 0; i < DI - 1; i++)
        for (long j = 0; j < DJ; j++)
            for (long k = 0; k < DK - 1; k++)
                surfaceAndCenter(D(i, j, k), D(i, j, k + 1), D(i + 1, j, k + 1), D(i + 1, j, k),
                                 surf_[1][faceIdx(1, i, j, k)], ctr_[1][faceIdx(1, i, j, k)]);
    for (long i = 0; i < DI - 1; i++)
        for (long j = 0; j < DJ - 1; j++)
            for (long k = 0; k < DK; k++)
                surfaceAndCenter(D(i, j, k), D(i + 1, j, k), D(i + 1, j + 1, k), D(i, j + 1, k),
                                 surf_[2][faceIdx(2, i, j, k)], ctr_[2][faceIdx(2, i, j, k)]);
}

// Mesh::computeFiniteVolumes (src/mesh.cpp:192-230): divergence theorem, x part.
void Mesh::finiteVolumes() {
    vol_.assign(nodes(), 0.0);
    for (long i = 0; i < ni_; i++)
        for (long j = 0; j < nj_; j++)
            for (long k = 0; k < nk_; k++) {
                const Vec3 s[6] = {-surf_[0][faceIdx(0, i, j, k)], -surf_[1][faceIdx(1, i, j, k)],
                                   -surf_[2][faceIdx(2, i, j, k)], surf_[0][faceIdx(0, i + 1, j, k)],
                                   surf_[1][faceIdx(1, i, j + 1, k)], surf_[2][faceIdx(2, i, j, k + 1)]};
                const Vec3 c[6] = {ctr_[0][faceIdx(0, i, j, k)], ctr_[1][faceIdx(1, i, j, k)],
                                   ctr_[2][faceIdx(2, i, j, k)], ctr_[0][faceIdx(0, i + 1, j, k)],
                                   ctr_[1][faceIdx(1, i, j + 1, k)], ctr_[2][faceIdx(2, i, j, k + 1)]};
                double v = 0.0;
                for (int f = 0; f < 6; f++) v += s[f].x * c[f].x;
                vol_[idx(i, j, k)] = v;
            }
}

// computeGradientGreenGauss with interpolateScalar (src/math_utils.cpp:173-234,
// 395-463) applied to the blockage (src/mesh.cpp:571-581).
void Mesh::blockageGradientGreenGauss() {
    const std::vector<double>& b = field("blockage");
    gradb_.assign(nodes(), Vec3());
    auto interp = [&](long i, long j, long k, const Vec3& pt, int dir) {
        const Vec3& p0 = vert_[idx(i, j, k)];
        const double f0 = b[idx(i, j, k)];
        long i1 = i, j1 = j, k1 = k;
        switch (dir) {
            case 0: if (i == 0) return f0; i1 = i - 1; break;
            case 1: if (i == ni_ - 1) return f0; i1 = i + 1; break;
            case 2: if (j == nj_ - 1) return f0; j1 = j + 1; break;
            case 3: if (j == 0) return f0; j1 = j - 1; break;
            case 4: if (k == 0) return f0; k1 = k - 1; break;
            default: if (k == nk_ - 1) return f0; k1 = k + 1; break;
        }
        const Vec3& p1 = vert_[idx(i1, j1, k1)];
        const double f1 = b[idx(i1, j1, k1)];
        const double d0 = (pt - p0).magnitude(), d1 = (pt - p1).magnitude();
        return f0 + (f1 - f0) * d0 / (d0 + d1);
    };
    for (long i = 0; i < ni_; i++)
        for (long j = 0; j < nj_; j++)
            for (long k = 0; k < nk_; k++) {
                const Vec3 s[6] = {-surf_[0][faceIdx(0, i, j, k)], surf_[0][faceIdx(0, i + 1, j, k)],
                                   surf_[1][faceIdx(1, i, j + 1, k)], -surf_[1][faceIdx(1, i, j, k)],
                                   -surf_[2][faceIdx(2, i, j, k)], surf_[2][faceIdx(2, i, j, k + 1)]};
                const Vec3 c[6] = {ctr_[0][faceIdx(0, i, j, k)], ctr_[0][faceIdx(0, i + 1, j, k)],
                                   ctr_[1][faceIdx(1, i, j + 1, k)], ctr_[1][faceIdx(1, i, j, k)],
                                   ctr_[2][faceIdx(2, i, j, k)], ctr_[2][faceIdx(2, i, j, k + 1)]};
                Vec3 g(0.0, 0.0, 0.0);
                for (int f = 0; f < 6; f++) g = g + s[f] * interp(i, j, k, c[f], f);
                gradb_[idx(i, j, k)] = g / vol_[idx(i, j, k)];
            }
}

// Mesh::checkPeriodicity (src/mesh.cpp:584-619) with atan2FromZeroTo2pi
// (src/math_utils.cpp:466-471).
void Mesh::checkPeriodicity(double translation, double angle) const {
    const Vec3 drag(0.0, 0.0, translation);
    auto atan2pos = [](double y, double x) {
        double a = std::atan2(y, x);
        if (a < 0) a += 2 * M_PI;
        return a;
    };
    for (long i = 0; i < ni_; i++)
        for (long j = 0; j < nj_; j++) {
            const Vec3& a = vert_[idx(i, j, 0)];
            const Vec3 b = vert_[idx(i, j, nk_ - 1)] - drag;
            const double dth = std::fmod(atan2pos(b.z, b.y) - atan2pos(a.z, a.y), 2.0 * M_PI);
            if (std::abs(dth - angle) > 1E-4)
                throw ConfigError("Periodicity check failed at (i,j)=(" + std::to_string(i) + "," + std::to_string(j) + ")");
            if (std::abs(translation) > 1e-6 && angle == 0.0 && std::abs(b.z - a.z) > 1E-4)
                throw ConfigError("Axial translation mismatch at (i,j)=(" + std::to_string(i) + "," + std::to_string(j) + ")");
        }
}

}  // namespace ctbfm
