// Restart: see restart.hpp.
#include "restart.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>

namespace ctbfm {

namespace {

std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return std::string();
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// atan2FromZeroTo2pi (src/math_utils.cpp:465-470)
double angle0to2pi(double y, double x) {
    double a = std::atan2(y, x);
    if (a < 0) a += 2 * M_PI;
    return a;
}

// rotateVectorAlongXAxis (src/math_utils.cpp:109-115)
Vec3 rotateX(const Vec3& v, double theta) {
    return Vec3(v.x, v.y * std::cos(theta) - v.z * std::sin(theta), v.y * std::sin(theta) + v.z * std::cos(theta));
}

// Nearest-point search over a static point set: a k-d tree whose node is the
// median along axis depth % D of its range (std::nth_element on that
// coordinate) and whose search descends the near side first, takes strictly
// closer points only and visits the far side only when the splitting plane is
// strictly closer than the best distance. Exact distance ties therefore
// resolve to the same point as the reference's KDTree (include/kdtree.hpp),
// which matters on refined grids whose nodes sit half-way between coarse ones.
template <int D>
class KdTree {
public:
    using Point = std::array<double, D>;

    explicit KdTree(const std::vector<Point>& pts) {
        std::vector<Entry> items(pts.size());
        for (size_t q = 0; q < pts.size(); q++) items[q] = Entry{pts[q], q};
        nodes_.reserve(pts.size());
        root_ = build(items, 0, items.size(), 0);
    }

    size_t nearest(const Point& x) const {
        size_t best = nodes_[static_cast<size_t>(root_)].orig;
        double bestD2 = std::numeric_limits<double>::max();
        search(root_, x, best, bestD2);
        return best;
    }

private:
    struct Entry {
        Point p;
        size_t orig;
    };
    struct Node {
        Point p;
        size_t orig;
        int axis, lo, hi;
    };
    std::vector<Node> nodes_;
    int root_ = -1;

    int build(std::vector<Entry>& items, size_t a, size_t b, int depth) {
        if (a >= b) return -1;
        const int axis = depth % D;
        const size_t mid = a + (b - a) / 2;
        std::nth_element(items.begin() + static_cast<long>(a), items.begin() + static_cast<long>(mid),
                         items.begin() + static_cast<long>(b),
                         [axis](const Entry& u, const Entry& v) { return u.p[axis] < v.p[axis]; });
        const int id = static_cast<int>(nodes_.size());
        nodes_.push_back(Node{items[mid].p, items[mid].orig, axis, -1, -1});
        const int lo = build(items, a, mid, depth + 1);
        const int hi = build(items, mid + 1, b, depth + 1);
        nodes_[static_cast<size_t>(id)].lo = lo;
        nodes_[static_cast<size_t>(id)].hi = hi;
        return id;
    }

    void search(int id, const Point& x, size_t& best, double& bestD2) const {
        if (id < 0) return;
        const Node& n = nodes_[static_cast<size_t>(id)];
        double d2 = 0.0;
        for (int d = 0; d < D; d++) {
            const double t = x[d] - n.p[d];
            d2 += t * t;
        }
        if (d2 < bestD2) {
            bestD2 = d2;
            best = n.orig;
        }
        const double off = x[n.axis] - n.p[n.axis];
        search(off <= 0.0 ? n.lo : n.hi, x, best, bestD2);
        if (off * off < bestD2) search(off <= 0.0 ? n.hi : n.lo, x, best, bestD2);
    }
};

// Conservative state of one node from (rho, velocity, T), as the three
// restart initialisations form it: p = p(rho, T), e = e(p, rho),
// et = e + 0.5 * (u.u).
void setNode(std::array<std::vector<double>, 5>& U, long q, double rho, const Vec3& v, double T, const HostFluid& f) {
    U[0][q] = rho;
    U[1][q] = rho * v.x;
    U[2][q] = rho * v.y;
    U[3][q] = rho * v.z;
    const double p = f.pressure_rho_T(rho, T);
    const double e = f.staticEnergy_p_rho(p, rho);
    const double et = e + 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z);
    U[4][q] = rho * et;
}

}  // namespace

std::string restartPath(const Config& config) {
    if (!config.has("RESTART_SOLUTION_FILEPATH"))
        throw ConfigError("Not found value for key \"RESTART_SOLUTION_FILEPATH\" in configuration.");
    const std::string file = config.get("RESTART_SOLUTION_FILEPATH");
    if (!file.empty() && file[0] == '/') return file;
    return config.directory().empty() ? file : config.directory() + "/" + file;
}

RestartFile readRestartFile(const std::string& path, const HostFluid& fluid) {
    std::ifstream f(path);
    if (!f.is_open()) throw ConfigError("Failed to open restart file: " + path);
    RestartFile r;
    std::string line;
    long* dims[3] = {&r.ni, &r.nj, &r.nk};
    for (long* d : dims) {
        if (!std::getline(f, line) || line.find('=') == std::string::npos)
            throw ConfigError("Restart file " + path + " lacks its NI/NJ/NK lines");
        try {
            *d = std::stol(line.substr(line.find('=') + 1));
        } catch (const std::exception&) {
            throw ConfigError("Restart file " + path + ": bad dimension line \"" + trim(line) + "\"");
        }
        if (*d < 0) throw ConfigError("Restart file " + path + ": negative dimension");
    }
    if (!std::getline(f, line)) throw ConfigError("Restart file " + path + " lacks its header line");
    std::map<std::string, long> col;
    {
        std::istringstream hs(line);
        std::string name;
        long c = 0;
        while (std::getline(hs, name, ',')) col[trim(name)] = c++;
    }
    auto find = [&](const char* a, const char* b) -> long {
        if (col.count(a)) return col[a];
        if (b && col.count(b)) return col[b];
        return -1;
    };
    const long ix = find("x", "X"), iy = find("y", "Y"), iz = find("z", "Z");
    const bool coords = ix >= 0 && iy >= 0 && iz >= 0;
    long need[5];
    const char* names[5] = {"Density", "Velocity X", "Velocity Y", "Velocity Z", "Total Energy"};
    for (int v = 0; v < 5; v++) {
        need[v] = find(names[v], nullptr);
        if (need[v] < 0) throw ConfigError("Restart file " + path + " has no \"" + names[v] + "\" column");
    }
    const long n = r.ni * r.nj * r.nk;
    r.xyz.assign(static_cast<size_t>(n), Vec3());
    r.rho.assign(static_cast<size_t>(n), 0.0);
    r.vx = r.vy = r.vz = r.T = r.rho;
    long row = 0, i = 0, j = 0, k = 0;
    std::vector<double> vals;
    while (std::getline(f, line)) {
        if (trim(line).empty()) continue;
        if (row >= n) throw ConfigError("Restart file " + path + " has more rows than NI*NJ*NK");
        const std::string at = "(" + std::to_string(i) + "," + std::to_string(j) + "," + std::to_string(k) + ")";
        vals.clear();
        std::istringstream ss(line);
        std::string cell;
        while (std::getline(ss, cell, ',')) {
            double v;
            try {
                v = std::stod(cell);
            } catch (const std::exception&) {
                throw ConfigError("Corrupted restart file '" + path + "': unreadable value \"" + trim(cell) +
                                  "\" at row index " + at + ".");
            }
            if (std::isnan(v) || std::isinf(v))
                throw ConfigError("Corrupted restart file '" + path + "': NaN or Inf encountered at row index " + at +
                                  ".");
            vals.push_back(v);
        }
        const long nv = static_cast<long>(vals.size());
        for (int v = 0; v < 5; v++)
            if (need[v] >= nv) throw ConfigError("Restart file " + path + ": short row at index " + at);
        if (coords && ix < nv && iy < nv && iz < nv) r.xyz[row] = Vec3(vals[ix], vals[iy], vals[iz]);
        const double rho = vals[need[0]];
        const Vec3 u(vals[need[1]], vals[need[2]], vals[need[3]]);
        r.rho[row] = rho;
        r.vx[row] = u.x;
        r.vy[row] = u.y;
        r.vz[row] = u.z;
        r.T[row] = fluid.temperature_rho_u_et(rho, u, vals[need[4]]);
        row++;
        if (++k == r.nk) {
            k = 0;
            if (++j == r.nj) {
                j = 0;
                ++i;
            }
        }
    }
    if (row != n)
        throw ConfigError("Restart file " + path + " has " + std::to_string(row) + " rows, NI*NJ*NK = " +
                          std::to_string(n));
    return r;
}

void restartState(const Config& config, const Mesh& mesh, Topology topo, bool periodic, const HostFluid& fluid,
                  std::array<std::vector<double>, 5>& U) {
    const RestartFile r = readRestartFile(restartPath(config), fluid);
    const long NI = mesh.ni(), NJ = mesh.nj(), NK = mesh.nk();
    for (auto& a : U) a.assign(static_cast<size_t>(mesh.nodes()), 0.0);
    // Config::getRestartType (include/config.hpp:197): "None" when absent
    const std::string type = config.has("RESTART_TYPE") ? config.get("RESTART_TYPE") : "None";
    const auto& V = mesh.vertices();

    bool nearest = type == "nearest_neighbor" || type == "nearest_neighbor_axisymmetric";
    if (!nearest && (r.ni != NI || r.nj != NJ || r.nk != NK)) {
        if (r.ni == NI && r.nj == NJ && type == "axisymmetric") {
            // Solver::axisymmetricRestart (src/solver.cpp:1002-1035): the
            // k = 0 plane of the file, rotated about x to each node's angle
            for (long i = 0; i < NI; i++)
                for (long j = 0; j < NJ; j++)
                    for (long k = 0; k < NK; k++) {
                        const Vec3& v0 = V[mesh.idx(i, j, 0)];
                        const Vec3& vk = V[mesh.idx(i, j, k)];
                        const double rot = angle0to2pi(vk.z, vk.y) - angle0to2pi(v0.z, v0.y);
                        const long s = (i * r.nj + j) * r.nk;
                        const Vec3 vel = rotateX(Vec3(r.vx[s], r.vy[s], r.vz[s]), rot);
                        setNode(U, mesh.idx(i, j, k), r.rho[s], vel, r.T[s], fluid);
                    }
            return;
        }
        if (type == "standard")
            throw ConfigError("Restart file dimensions (" + std::to_string(r.ni) + "," + std::to_string(r.nj) + "," +
                              std::to_string(r.nk) + ") do not match solver dimensions (" + std::to_string(NI) + "," +
                              std::to_string(NJ) + "," + std::to_string(NK) +
                              ") and RESTART_TYPE=standard was requested.");
        nearest = true;
    }
    if (!nearest) {  // Solver::standardRestart (src/solver.cpp:968-1000)
        for (long q = 0; q < mesh.nodes(); q++)
            setNode(U, q, r.rho[q], Vec3(r.vx[q], r.vy[q], r.vz[q]), r.T[q], fluid);
        return;
    }
    // Solver::nearestNeighborRestart (src/solver.cpp:1037-1153)
    const long n = r.ni * r.nj * r.nk;
    if (n == 0) throw ConfigError("Cannot perform nearest-neighbor restart: restart data is empty.");
    const bool axi = type == "axisymmetric" || type == "nearest_neighbor_axisymmetric" ||
                     topo == Topology::Axisymmetric || (r.nk == 1 && NK > 1 && periodic);
    if (axi) {  // nearest in the meridional plane (x, r), velocity rotated to the node's angle
        std::vector<std::array<double, 2>> pts(static_cast<size_t>(n));
        for (long q = 0; q < n; q++) {
            const Vec3& p = r.xyz[q];
            pts[q] = {p.x, std::sqrt(p.y * p.y + p.z * p.z)};
        }
        const KdTree<2> tree(pts);
        for (long q = 0; q < mesh.nodes(); q++) {
            const Vec3& p = V[q];
            const double rt = std::sqrt(p.y * p.y + p.z * p.z);
            const double tt = angle0to2pi(p.z, p.y);
            const size_t b = tree.nearest({p.x, rt});
            const Vec3& pc = r.xyz[b];
            const double rot = tt - angle0to2pi(pc.z, pc.y);
            const Vec3 vel = rotateX(Vec3(r.vx[b], r.vy[b], r.vz[b]), rot);
            setNode(U, q, r.rho[b], vel, r.T[b], fluid);
        }
        return;
    }
    std::vector<std::array<double, 3>> pts(static_cast<size_t>(n));
    for (long q = 0; q < n; q++) pts[q] = {r.xyz[q].x, r.xyz[q].y, r.xyz[q].z};
    const KdTree<3> tree(pts);
    for (long q = 0; q < mesh.nodes(); q++) {
        const Vec3& p = V[q];
        const size_t b = tree.nearest({p.x, p.y, p.z});
        setNode(U, q, r.rho[b], Vec3(r.vx[b], r.vy[b], r.vz[b]), r.T[b], fluid);
    }
}

}  // namespace ctbfm
