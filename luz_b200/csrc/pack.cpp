// pack.cpp — flattens a LuzSceneDesc into the device arena layout (layout.h).
//
// The BVH builders reproduce the reference's algorithms exactly, in double and
// with the same standard-library algorithms, so that node topology, triangle
// order and top-level child order are identical to what the CPU renderer
// traverses:
//   mesh:  Mesh::_buildPackedBVH / _buildPackedBVHNode / findBinnedSAHSplit
//          (src/core/Hittables/Mesh.cpp:16-18, 217-306, 383-521): 12 bins, leaf
//          <= 8, minimum side max(1, n/16), std::partition on bin <= split,
//          std::nth_element median fallback on centroid (tie: box minimum);
//   top:   BVHNode::BVHNode (src/core/Hittables/BVHNode.cpp:142-185): std::sort
//          on box minimum of the largest-extent axis, median split, leaves of
//          <= 8 children (<= 16 at the root);
//   scene: Scene::updateAccelerationStructure (src/scene/Scene.cpp:655-688) and
//          Scene::updateLights (src/scene/Scene.cpp:615-638).
// The results are then rounded outward to FP32 (boxes) or to nearest (vertices).
#include <thread>
#include "pack.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <numeric>

namespace luz {

namespace {

thread_local std::string g_error;

constexpr double kTMin64 = 0.001;       // T_MIN
constexpr double kPi = 3.14159265358979323846;

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    explicit V3(const double* p) : x(p[0]), y(p[1]), z(p[2]) {}
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
// Vector3 operators of include/luz/Vector3.hpp (note: v / f is (1/f) * v).
inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(double f, V3 v) { return V3(f * v.x, f * v.y, f * v.z); }
inline V3 operator*(V3 v, double f) { return f * v; }
inline V3 operator/(V3 v, double f) { return (1.0 / f) * v; }
inline double dot(V3 a, V3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
inline V3 cross(V3 a, V3 b)
{
    return V3((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
inline double len2(V3 v) { return (v.x * v.x) + (v.y * v.y) + (v.z * v.z); }
inline V3 normalize(V3 v) { return v / std::sqrt(len2(v)); }
inline double luminance(const double* c) { return c[0] * 0.2722287168 + c[1] * 0.6740817658 + c[2] * 0.0536895174; }

float f_down(double x)
{
    float f = (float)x;
    if ((double)f > x) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    return f;
}
float f_up(double x)
{
    float f = (float)x;
    if ((double)f < x) f = std::nextafter(f, std::numeric_limits<float>::infinity());
    return f;
}
void put_box(const Box64& b, float* mn, float* mx)
{
    for (int a = 0; a < 3; a++) {
        mn[a] = f_down(b.mn[a]);
        mx[a] = f_up(b.mx[a]);
    }
}
void put3(float* d, V3 v)
{
    d[0] = (float)v.x;
    d[1] = (float)v.y;
    d[2] = (float)v.z;
}

[[noreturn]] void invalid(const std::string& m) { throw Status(LUZ_E_INVALID, m); }
[[noreturn]] void unsupported(const std::string& m) { throw Status(LUZ_E_UNSUPPORTED, m); }

bool finite3(const double* c) { return std::isfinite(c[0]) && std::isfinite(c[1]) && std::isfinite(c[2]); }
double clamp01(double v) { return std::isfinite(v) ? std::max(0.0, std::min(1.0, v)) : 0.0; }
double roughness_to_alpha(double r)  // BSDF::roughnessToAlpha (src/core/Materials/BSDF.cpp:53-57)
{
    r = clamp01(r);
    return std::max(1e-4, r * r);
}

// ----------------------------------------------------------------------------- materials

void check_unit(double v, const char* label)
{
    if (!std::isfinite(v) || v < 0.0 || v > 1.0) invalid(std::string(label) + " must be finite and in [0,1].");
}

// IESProfile::candelaAt (IESProfile.cpp:231-299): bilinear in (vertical,
// horizontal) degrees, zero outside the vertical range, horizontal angles
// wrapped to [0, 360) and closed over the last interval.
double ies_candela(const double* va, int nv, const double* ha, int nh, const double* cd, double vdeg, double hdeg)
{
    if (nv <= 0 || nh <= 0 || !std::isfinite(vdeg)) return 0.0;
    if (vdeg < va[0] || vdeg > va[nv - 1]) return 0.0;
    int v0 = 0;
    while (v0 + 1 < nv && va[v0 + 1] < vdeg) v0++;
    const int v1 = std::min(v0 + 1, nv - 1);
    const double vspan = va[v1] - va[v0];
    const double vt = vspan > 0.0 ? (vdeg - va[v0]) / vspan : 0.0;
    int h0 = 0, h1 = 0;
    double ht = 0.0;
    if (nh > 1) {
        double hz = std::isfinite(hdeg) ? std::fmod(hdeg, 360.0) : 0.0;
        if (hz < 0.0) hz += 360.0;
        const double first = ha[0], last = ha[nh - 1];
        if (hz < first) hz += 360.0;
        if (hz > last && last >= 360.0) hz = std::min(hz, last);
        while (h0 + 1 < nh && ha[h0 + 1] < hz) h0++;
        if (h0 + 1 < nh) {
            h1 = h0 + 1;
            const double hspan = ha[h1] - ha[h0];
            ht = hspan > 0.0 ? (hz - ha[h0]) / hspan : 0.0;
        } else {
            h1 = 0;
            const double hspan = (first + 360.0) - ha[h0];
            ht = hspan > 0.0 ? (hz - ha[h0]) / hspan : 0.0;
        }
    }
    auto lerp = [](double a, double b, double t) { return a * (1.0 - t) + b * t; };
    return lerp(lerp(cd[h0 * nv + v0], cd[h0 * nv + v1], vt), lerp(cd[h1 * nv + v0], cd[h1 * nv + v1], vt), ht);
}

// integrateTotalLumens (IESProfile.cpp:111-131): midpoint rule on 180 x 360 cells.
double ies_flux(const double* va, int nv, const double* ha, int nh, const double* cd)
{
    const double dth = kPi / 180.0, dph = (2.0 * kPi) / 360.0;
    double total = 0.0;
    for (int v = 0; v < 180; v++) {
        const double th = ((double)v + 0.5) * dth;
        const double vdeg = th * (180.0 / kPi);
        const double st = std::sin(th);
        for (int h = 0; h < 360; h++) {
            const double hdeg = ((double)h + 0.5) * 360.0 / 360.0;
            total += ies_candela(va, nv, ha, nh, cd, vdeg, hdeg) * st * dth * dph;
        }
    }
    return total;
}

GMaterial pack_material(const LuzMaterialDesc& m, int texture_count)
{
    GMaterial g{};
    g.type = m.type;
    g.texture = m.texture;
    if (m.texture >= texture_count || m.texture < -1) invalid("Material texture index out of range.");
    g.rtexture = -1;
    if (m.has_roughness_texture) {   // an extension: the reference's Metal roughness is a scalar
        if (m.type != LUZ_MAT_METAL) invalid("Roughness textures are defined for Metal materials only.");
        if (m.roughness_texture < 0 || m.roughness_texture >= texture_count)
            invalid("Roughness texture index out of range.");
        g.rtexture = m.roughness_texture;
    }
    for (int a = 0; a < 3; a++) {
        g.color[a] = (float)m.color[a];
        g.eta[a] = (float)m.eta[a];
        g.k[a] = (float)m.k[a];
        g.absorption[a] = (float)m.absorption[a];
        g.ss_radius_m[a] = (float)(m.subsurface_radius[a] * m.subsurface_scale);
        g.ss_color[a] = (float)clamp01(m.subsurface_color[a]);
        g.gcolor[a] = (float)m.glossy_color[a];
    }
    g.gweight = (float)m.glossy_weight;
    g.roughness = (float)m.roughness;
    g.alpha = (float)roughness_to_alpha(m.roughness);
    g.clearcoat_alpha = (float)roughness_to_alpha(m.clearcoat_roughness);
    g.ior = (float)m.ior;
    g.anisotropy = (float)m.anisotropy;
    g.metallic = (float)m.metallic;
    g.transmission = (float)m.transmission;
    g.clearcoat = (float)m.clearcoat;
    g.clearcoat_roughness = (float)m.clearcoat_roughness;
    g.sheen = (float)m.sheen;
    g.subsurface = (float)m.subsurface;
    {
        const double r0 = (m.ior - 1.0) / (m.ior + 1.0);
        g.f0_diel = (float)clamp01(r0 * r0);
    }
    const bool absorb = m.absorption[0] > 0.0 || m.absorption[1] > 0.0 || m.absorption[2] > 0.0;
    switch (m.type) {
    case LUZ_MAT_LAMBERTIAN:
    case LUZ_MAT_EMISSIVE:
        break;
    case LUZ_MAT_ISOTROPIC:
        g.flags |= MF_CAN_TRANSMIT;   // materialCanTransmitThroughGeometry (ColorHelper.cpp:327-355)
        break;
    case LUZ_MAT_HENYEY_GREENSTEIN:
        if (!std::isfinite(m.anisotropy) || m.anisotropy < -0.99 || m.anisotropy > 0.99)
            invalid("Volume anisotropy must be finite and between -0.99 and 0.99.");
        g.flags |= MF_CAN_TRANSMIT;
        break;
    case LUZ_MAT_METAL:
        if (!std::isfinite(m.roughness) || m.roughness < 0.0 || m.roughness > 1.0)
            invalid("Metal roughness must be finite and in [0,1].");
        if (m.conductor) {
            for (int a = 0; a < 3; a++) {
                if (!std::isfinite(m.eta[a]) || m.eta[a] <= 0.0)
                    invalid("Conductor eta must have finite positive channels.");
                if (!std::isfinite(m.k[a]) || m.k[a] < 0.0)
                    invalid("Conductor extinction coefficient must have finite non-negative channels.");
            }
            g.flags |= MF_CONDUCTOR;
        }
        g.flags |= MF_TRANSPORT;
        break;
    case LUZ_MAT_DIELECTRIC:
        if (!std::isfinite(m.ior) || m.ior <= 0.0) invalid("Dielectric refractive index must be finite and positive.");
        if (!std::isfinite(m.roughness) || m.roughness < 0.0 || m.roughness > 1.0)
            invalid("Dielectric roughness must be finite and in [0,1].");
        if (!finite3(m.absorption) || m.absorption[0] < 0 || m.absorption[1] < 0 || m.absorption[2] < 0)
            invalid("Dielectric absorption coefficient must have finite non-negative channels.");
        g.flags |= MF_CAN_TRANSMIT | MF_TRANSPORT;
        if (absorb) g.flags |= MF_ABSORPTION;
        break;
    case LUZ_MAT_PRINCIPLED:
        check_unit(m.metallic, "Principled metallic");
        check_unit(m.roughness, "Principled roughness");
        check_unit(m.transmission, "Principled transmission");
        if (!std::isfinite(m.ior) || m.ior <= 0.0) invalid("Principled refractive index must be finite and positive.");
        check_unit(m.clearcoat, "Principled clearcoat");
        check_unit(m.clearcoat_roughness, "Principled clearcoat roughness");
        check_unit(m.sheen, "Principled sheen");
        check_unit(m.subsurface, "Principled subsurface");
        if (m.subsurface_method != 0 && m.subsurface_method != 1) invalid("Unknown principled subsurface method.");
        if (m.subsurface_method == 1) g.flags |= MF_THIN;
        if (m.transmission > 0.0 || (m.subsurface > 0.0 && m.subsurface_method == 1)) g.flags |= MF_CAN_TRANSMIT;
        if (m.transmission > 0.0 && absorb) g.flags |= MF_ABSORPTION;
        if (m.metallic <= 1e-6 && m.roughness <= 1e-4 && m.transmission >= 1.0 - 1e-6 && m.clearcoat <= 1e-6
            && m.sheen <= 1e-6 && m.subsurface <= 1e-6)
            g.flags |= MF_SMOOTH_FULL_TRANSMISSION;
        if (m.metallic >= 0.5 || m.transmission > 0.05 || m.clearcoat > 0.5) g.flags |= MF_TRANSPORT;
        break;
    case LUZ_MAT_GLOSSY:
        check_unit(m.roughness, "Glossy roughness");
        break;
    case LUZ_MAT_DIFFUSE_GLOSSY:
        check_unit(m.glossy_weight, "Diffuse-glossy weight");
        check_unit(m.roughness, "Diffuse-glossy roughness");
        break;
    default:
        unsupported("Material type " + std::to_string(m.type) + " is not on the GPU path.");
    }
    return g;
}

// ----------------------------------------------------------------------------- mesh BVH (exact)

constexpr std::size_t kLeafSize = 8;      // MESH_BVH_LEAF_SIZE
constexpr std::size_t kBins = 12;         // MESH_BVH_SAH_BINS
constexpr double kCentroidEps = 1e-12;    // MESH_BVH_CENTROID_EPSILON

Box64 merge(const Box64& a, const Box64& b)  // mergeBoxes (Mesh.cpp:51-65)
{
    Box64 r;
    for (int i = 0; i < 3; i++) {
        r.mn[i] = std::min(a.mn[i], b.mn[i]);
        r.mx[i] = std::max(a.mx[i], b.mx[i]);
    }
    return r;
}
Box64 merge_f(const Box64& a, const Box64& b)  // Utilities::mergeBoundingBoxes (fmin/fmax)
{
    Box64 r;
    for (int i = 0; i < 3; i++) {
        r.mn[i] = std::fmin(a.mn[i], b.mn[i]);
        r.mx[i] = std::fmax(a.mx[i], b.mx[i]);
    }
    return r;
}
double box_area(const Box64& b)
{
    const double x = std::max(0.0, b.mx[0] - b.mn[0]);
    const double y = std::max(0.0, b.mx[1] - b.mn[1]);
    const double z = std::max(0.0, b.mx[2] - b.mn[2]);
    return 2.0 * ((x * y) + (x * z) + (y * z));
}
int largest_axis(const Box64& b)
{
    const double ex = b.mx[0] - b.mn[0], ey = b.mx[1] - b.mn[1], ez = b.mx[2] - b.mn[2];
    if (ex >= ey && ex >= ez) return 0;
    if (ey >= ez) return 1;
    return 2;
}
std::size_t bin_for(double c, double mn, double scale)
{
    std::size_t b = static_cast<std::size_t>((c - mn) * scale);
    return b >= kBins ? kBins - 1 : b;
}

struct Bin {
    Box64 box{};
    std::size_t count = 0;
    bool has = false;
};

struct MeshBuilder {
    const std::vector<Box64>& boxes;
    const std::vector<V3>& cent;
    std::vector<std::size_t>& idx;   // triangle order, partitioned in place (shared by sub-builders)
    std::vector<LuzMeshNode64>& out;
    int max_depth = 0;

    struct Split {
        bool found = false;
        int axis = 0;
        std::size_t split = 0;
        double cmin = 0, scale = 0;
    };

    // The best split on one axis (cost, bin, range), as the reference's loop over that
    // axis's bins finds it: strictly lower cost wins, so the first bin of equal cost stays.
    Split axis_split(std::size_t s, std::size_t e, int axis, double& best_cost) const
    {
        const std::size_t n = e - s;
        const std::size_t min_side = std::max<std::size_t>(1, n / 16);
        Split best;
        best_cost = std::numeric_limits<double>::infinity();
        double cmin = std::numeric_limits<double>::infinity();
        double cmax = -std::numeric_limits<double>::infinity();
        for (std::size_t i = s; i < e; i++) {
            const double c = cent[idx[i]][axis];
            cmin = std::min(cmin, c);
            cmax = std::max(cmax, c);
        }
        const double ext = cmax - cmin;
        if (ext <= kCentroidEps) return best;
        const double scale = static_cast<double>(kBins) / ext;
        std::array<Bin, kBins> bins;
        for (std::size_t i = s; i < e; i++) {
            const std::size_t t = idx[i];
            Bin& b = bins[bin_for(cent[t][axis], cmin, scale)];
            b.box = b.has ? merge(b.box, boxes[t]) : boxes[t];
            b.count++;
            b.has = true;
        }
        std::array<Bin, kBins> left, right;
        Bin rl, rr;
        auto mergeBin = [](Bin& t, const Bin& src) {
            if (!src.has) return;
            t.box = t.has ? merge(t.box, src.box) : src.box;
            t.count += src.count;
            t.has = true;
        };
        for (std::size_t i = 0; i < kBins; i++) {
            mergeBin(rl, bins[i]);
            left[i] = rl;
        }
        for (std::size_t i = kBins; i > 0; i--) {
            mergeBin(rr, bins[i - 1]);
            right[i - 1] = rr;
        }
        for (std::size_t sb = 0; sb + 1 < kBins; sb++) {
            const Bin& l = left[sb];
            const Bin& r = right[sb + 1];
            if (!l.has || !r.has || l.count < min_side || r.count < min_side) continue;
            const double cost = (box_area(l.box) * static_cast<double>(l.count))
                                + (box_area(r.box) * static_cast<double>(r.count));
            if (cost < best_cost) {
                best_cost = cost;
                best.found = true;
                best.axis = axis;
                best.split = sb;
                best.cmin = cmin;
                best.scale = scale;
            }
        }
        return best;
    }

    // findBinnedSAHSplit: the axes in order, a strictly lower cost replacing the best so
    // far. Large ranges evaluate the three axes on threads and then compare them in the
    // same order, which picks the same split.
    Split find_split(std::size_t s, std::size_t e) const
    {
        Split per[3];
        double cost[3];
        if (e - s >= (std::size_t(1) << 17)) {
            std::thread t1([&] { per[1] = axis_split(s, e, 1, cost[1]); });
            std::thread t2([&] { per[2] = axis_split(s, e, 2, cost[2]); });
            per[0] = axis_split(s, e, 0, cost[0]);
            t1.join();
            t2.join();
        } else {
            for (int a = 0; a < 3; a++) per[a] = axis_split(s, e, a, cost[a]);
        }
        Split best;
        double best_cost = std::numeric_limits<double>::infinity();
        for (int a = 0; a < 3; a++)
            if (per[a].found && cost[a] < best_cost) {
                best_cost = cost[a];
                best = per[a];
            }
        return best;
    }

    std::size_t build(std::size_t s, std::size_t e, int depth)
    {
        max_depth = std::max(max_depth, depth);
        const std::size_t node = out.size();
        const std::size_t n = e - s;
        Box64 nb{};
        bool has = false;
        for (std::size_t i = s; i < e; i++) {
            nb = has ? merge(nb, boxes[idx[i]]) : boxes[idx[i]];
            has = true;
        }
        out.push_back(LuzMeshNode64{});
        for (int a = 0; a < 3; a++) {
            out[node].bmin[a] = nb.mn[a];
            out[node].bmax[a] = nb.mx[a];
        }
        if (n <= kLeafSize) {
            out[node].start = (int64_t)s;
            out[node].count = (int64_t)n;
            out[node].is_leaf = 1;
            return node;
        }
        const Split sp = find_split(s, e);
        std::size_t mid = s;
        if (sp.found) {
            auto it = std::partition(idx.begin() + s, idx.begin() + e, [&](std::size_t t) {
                return bin_for(cent[t][sp.axis], sp.cmin, sp.scale) <= sp.split;
            });
            mid = static_cast<std::size_t>(it - idx.begin());
        }
        if (mid == s || mid == e) {
            const int axis = largest_axis(nb);
            mid = s + n / 2;
            std::nth_element(idx.begin() + s, idx.begin() + mid, idx.begin() + e, [&](std::size_t a, std::size_t b) {
                const double ca = cent[a][axis], cb = cent[b][axis];
                if (ca == cb) return boxes[a].mn[axis] < boxes[b].mn[axis];
                return ca < cb;
            });
        }
        const std::size_t l = build(s, mid, depth + 1);
        const std::size_t r = build(mid, e, depth + 1);
        out[node].left = (int64_t)l;
        out[node].right = (int64_t)r;
        return node;
    }

    // The same build, with the two subtrees of the top `par` levels built on two
    // threads: each subtree goes to a vector of its own (node numbers from 0) and is
    // appended after its parent in build's order (the node, its left subtree, its right
    // subtree), its child numbers shifted by where it lands. Subtrees own disjoint
    // ranges of idx. The nodes, their numbers and the triangle order are build's.
    std::size_t build_parallel(std::size_t s, std::size_t e, int depth, int par)
    {
        const std::size_t n = e - s;
        if (par <= 0 || n < (std::size_t(1) << 15)) return build(s, e, depth);
        max_depth = std::max(max_depth, depth);
        const std::size_t node = out.size();
        Box64 nb{};
        bool has = false;
        for (std::size_t i = s; i < e; i++) {
            nb = has ? merge(nb, boxes[idx[i]]) : boxes[idx[i]];
            has = true;
        }
        out.push_back(LuzMeshNode64{});
        for (int a = 0; a < 3; a++) {
            out[node].bmin[a] = nb.mn[a];
            out[node].bmax[a] = nb.mx[a];
        }
        const Split sp = find_split(s, e);
        std::size_t mid = s;
        if (sp.found) {
            auto it = std::partition(idx.begin() + s, idx.begin() + e, [&](std::size_t t) {
                return bin_for(cent[t][sp.axis], sp.cmin, sp.scale) <= sp.split;
            });
            mid = static_cast<std::size_t>(it - idx.begin());
        }
        if (mid == s || mid == e) {
            const int axis = largest_axis(nb);
            mid = s + n / 2;
            std::nth_element(idx.begin() + s, idx.begin() + mid, idx.begin() + e, [&](std::size_t a, std::size_t b) {
                const double ca = cent[a][axis], cb = cent[b][axis];
                if (ca == cb) return boxes[a].mn[axis] < boxes[b].mn[axis];
                return ca < cb;
            });
        }
        std::vector<LuzMeshNode64> lo, hi;
        MeshBuilder L{boxes, cent, idx, lo, 0}, R{boxes, cent, idx, hi, 0};
        std::thread t([&] { L.build_parallel(s, mid, depth + 1, par - 1); });
        R.build_parallel(mid, e, depth + 1, par - 1);
        t.join();
        max_depth = std::max(max_depth, std::max(L.max_depth, R.max_depth));
        auto append = [&](const std::vector<LuzMeshNode64>& sub) {
            const int64_t base = (int64_t)out.size();
            for (LuzMeshNode64 nd : sub) {
                if (!nd.is_leaf) {
                    nd.left += base;
                    nd.right += base;
                }
                out.push_back(nd);
            }
            return base;
        };
        out[node].left = append(lo);
        out[node].right = append(hi);
        return node;
    }
};

void build_mesh(const LuzMeshDesc& m, MeshBuild& mb)
{
    if (m.triangle_count < 0 || (m.triangle_count > 0 && !m.positions)) invalid("Mesh positions are missing.");
    mb.material = m.material;
    const std::size_t tc = (std::size_t)m.triangle_count;
    mb.vtx.reserve(9 * tc);
    mb.v0.reserve(3 * tc);
    mb.e1.reserve(3 * tc);
    mb.e2.reserve(3 * tc);
    mb.fn.reserve(3 * tc);
    mb.area.reserve(tc);
    if (m.normals) {
        mb.has_vn.reserve(tc);
        mb.vn.reserve(9 * tc);
    }
    if (m.uvs) mb.uv.reserve(6 * tc);
    for (int64_t t = 0; t < m.triangle_count; t++) {
        const double* p = m.positions + 9 * t;
        const V3 a(p), b(p + 3), c(p + 6);
        const V3 e1 = b - a, e2 = c - a;
        const V3 gn = cross(e1, e2);
        const double nls = len2(gn);
        if (nls <= 1e-24) continue;                         // _isDegenerate -> area 0 -> removed
        const double nl = std::sqrt(nls);
        const double area = nl / 2.0;
        if (area <= 0.0) continue;
        const V3 fn = gn / nl;
        for (int k = 0; k < 9; k++) mb.vtx.push_back(p[k]);
        for (int k = 0; k < 3; k++) {
            mb.v0.push_back(a[k]);
            mb.e1.push_back(e1[k]);
            mb.e2.push_back(e2[k]);
            mb.fn.push_back(fn[k]);
        }
        mb.area.push_back(area);
        if (m.normals) {
            const double* n = m.normals + 9 * t;
            const bool ok = len2(V3(n)) > 1e-24 && len2(V3(n + 3)) > 1e-24 && len2(V3(n + 6)) > 1e-24;
            mb.has_vn.push_back(ok ? 1 : 0);
            for (int k = 0; k < 9; k++) mb.vn.push_back(n[k]);
        }
        if (m.uvs) {
            const double* u = m.uvs + 6 * t;
            for (int k = 0; k < 6; k++) mb.uv.push_back(u[k]);
        }
    }
    const std::size_t n = mb.area.size();
    double total = 0.0;
    for (std::size_t i = 0; i < n; i++) total += mb.area[i];
    mb.total_area = total;
    if (n == 0) return;
    std::vector<Box64> boxes(n);
    std::vector<V3> cent(n);
    // Triangle boxes from the stored vertices (Triangle::_updateCache, Triangle.cpp:110-125).
    std::size_t k = 0;
    for (int64_t t = 0; t < m.triangle_count; t++) {
        const double* p = m.positions + 9 * t;
        const V3 a(p), b(p + 3), c(p + 6);
        const V3 gn = cross(b - a, c - a);
        const double nls = len2(gn);
        if (nls <= 1e-24 || std::sqrt(nls) / 2.0 <= 0.0) continue;
        Box64& bx = boxes[k];
        bx.mn[0] = std::min(a.x, std::min(b.x, c.x)) - kTMin64;
        bx.mn[1] = std::min(a.y, std::min(b.y, c.y)) - kTMin64;
        bx.mn[2] = std::min(a.z, std::min(b.z, c.z)) - kTMin64;
        bx.mx[0] = std::max(a.x, std::max(b.x, c.x)) + kTMin64;
        bx.mx[1] = std::max(a.y, std::max(b.y, c.y)) + kTMin64;
        bx.mx[2] = std::max(a.z, std::max(b.z, c.z)) + kTMin64;
        const V3 mn(bx.mn[0], bx.mn[1], bx.mn[2]), mx(bx.mx[0], bx.mx[1], bx.mx[2]);
        cent[k] = (mn + mx) / 2.0;
        k++;
    }
    std::vector<std::size_t> idx(n);
    std::iota(idx.begin(), idx.end(), std::size_t(0));
    MeshBuilder b{boxes, cent, idx, mb.nodes, 0};
    mb.nodes.reserve(2 * n);
    b.build_parallel(0, n, 0, 3);   // up to 8 subtrees built at once
    mb.depth = b.max_depth;
    mb.order.assign(idx.begin(), idx.end());
    for (int a = 0; a < 3; a++) {
        mb.box.mn[a] = mb.nodes[0].bmin[a];
        mb.box.mx[a] = mb.nodes[0].bmax[a];
    }
}

// ----------------------------------------------------------------------------- object boxes

struct RectBasis {
    V3 n, wa, ha;
};

// Rectangle::_buildBasis with defaultRectangleBasis / normalizedProjectedAxis
// (src/core/Hittables/Rectangle.cpp:14-66, 127-152).
bool rect_basis(const LuzObjectDesc& o, RectBasis& rb)
{
    const V3 orient(o.orientation);
    if (len2(orient) <= 0.0) return false;
    rb.n = normalize(orient);
    const V3 n = rb.n;
    if (std::fabs(n.y) > 0.999) {
        rb.wa = V3(1, 0, 0);
        rb.ha = V3(0, 0, 1);
    } else if (std::fabs(n.z) > 0.999) {
        rb.wa = V3(1, 0, 0);
        rb.ha = V3(0, 1, 0);
    } else if (std::fabs(n.x) > 0.999) {
        rb.wa = V3(0, 0, 1);
        rb.ha = V3(0, 1, 0);
    } else {
        V3 helper(0, 1, 0);
        if (std::fabs(dot(helper, n)) > 0.9) helper = V3(1, 0, 0);
        rb.wa = normalize(cross(helper, n));
        rb.ha = normalize(cross(n, rb.wa));
    }
    const bool has_axes = o.has_axes && len2(V3(o.width_axis)) > 1e-24 && len2(V3(o.height_axis)) > 1e-24;
    if (!has_axes) return true;
    auto proj = [&](V3 axis, V3& out) {
        axis = axis - (n * dot(axis, n));
        if (len2(axis) <= 1e-24) return false;
        out = normalize(axis);
        return true;
    };
    if (!proj(V3(o.width_axis), rb.wa)) return false;
    if (!proj(V3(o.height_axis), rb.ha)) return false;
    rb.ha = rb.ha - (rb.wa * dot(rb.ha, rb.wa));
    if (len2(rb.ha) <= 1e-24) return false;
    rb.ha = normalize(rb.ha);
    return true;
}

bool rect_box(const V3& pos, const RectBasis& rb, double w, double h, Box64& out)
{
    const double hw = w / 2.0, hh = h / 2.0;
    const V3 c0 = pos + (rb.wa * hw) + (rb.ha * hh);
    const V3 c1 = pos + (rb.wa * hw) - (rb.ha * hh);
    const V3 c2 = pos - (rb.wa * hw) + (rb.ha * hh);
    const V3 c3 = pos - (rb.wa * hw) - (rb.ha * hh);
    for (int a = 0; a < 3; a++) {
        out.mn[a] = std::min(std::min(c0[a], c1[a]), std::min(c2[a], c3[a]));
        out.mx[a] = std::max(std::max(c0[a], c1[a]), std::max(c2[a], c3[a]));
        if (std::fabs(out.mx[a] - out.mn[a]) <= kTMin64) {
            out.mn[a] -= kTMin64;
            out.mx[a] += kTMin64;
        }
    }
    return true;
}

GRect make_rect(const V3& pos, const RectBasis& rb, double w, double h)
{
    GRect r{};
    put3(r.p, pos);
    put3(r.n, rb.n);
    put3(r.wa, rb.wa);
    put3(r.ha, rb.ha);
    r.hw = (float)(w / 2.0);
    r.hh = (float)(h / 2.0);
    r.w = (float)w;
    r.h = (float)h;
    return r;
}

// MeshInstance::InstanceTransform (src/core/Hittables/MeshInstance.cpp:48-167).
struct Xform {
    V3 pos, scale;
    double cx, sx, cy, sy, cz, sz;
    bool invertible, uniform;
    double uniform_scale;
    Xform(const LuzObjectDesc& o)
    {
        const double d2r = 3.14159265358979323846 / 180.0;
        pos = V3(o.position);
        scale = V3(o.scale);
        const double xr = o.rotation_degrees[0] * d2r, yr = o.rotation_degrees[1] * d2r, zr = o.rotation_degrees[2] * d2r;
        const double ax = std::fabs(scale.x), ay = std::fabs(scale.y), az = std::fabs(scale.z);
        cx = std::cos(xr);
        sx = std::sin(xr);
        cy = std::cos(yr);
        sy = std::sin(yr);
        cz = std::cos(zr);
        sz = std::sin(zr);
        invertible = ax > 1e-12 && ay > 1e-12 && az > 1e-12;
        uniform = std::fabs(ax - ay) <= 1e-12 && std::fabs(ax - az) <= 1e-12;
        uniform_scale = uniform ? ax * ax : 1.0;
    }
    V3 rotate(V3 v) const
    {
        double x = v.x, y = v.y, z = v.z;
        double ny = (y * cx) - (z * sx);
        double nz = (y * sx) + (z * cx);
        y = ny;
        z = nz;
        double nx = (x * cy) + (z * sy);
        nz = (-x * sy) + (z * cy);
        x = nx;
        z = nz;
        nx = (x * cz) - (y * sz);
        ny = (x * sz) + (y * cz);
        return V3(nx, ny, z);
    }
    V3 point(V3 p) const { return rotate(V3(p.x * scale.x, p.y * scale.y, p.z * scale.z)) + pos; }
};

bool finite_v(V3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

}  // namespace

void set_error(const std::string& m) { g_error = m; }
const std::string& get_error() { return g_error; }

int64_t ScenePack::device_bytes() const
{
    return (int64_t)(rects.size() * sizeof(GRect) + objects.size() * sizeof(GObject)
                     + top_nodes.size() * sizeof(GTopNode) + top_children.size() * sizeof(GTopChild)
                     + nodes4.size() * sizeof(GNode4) + tris.size() * sizeof(GTri) + tri_shade.size() * sizeof(GTriShade)
                     + vnormals.size() * 4 + vuvs.size() * 4 + meshes.size() * sizeof(GMesh)
                     + materials.size() * sizeof(GMaterial) + textures.size() * sizeof(GTexture) + texels.size() * 4
                     + lights.size() * sizeof(GLight) + cdf.size() * 8 + index_pool.size() * 4 + env_texels.size() * 4);
}

GCamera prepare_camera(const LuzCameraDesc& c, double mpu, int width, int height)
{
    GCamera g{};
    const double W = (double)width, H = (double)height;
    g.inv_w1 = W > 1.0 ? 1.0 / (W - 1.0) : 0.0;
    g.inv_h1 = H > 1.0 ? 1.0 / (H - 1.0) : 0.0;
    const V3 pos(c.position);
    const double focus = c.focus_distance_m / mpu;
    double vw = focus * c.sensor_width_m / c.focal_length_m;
    double vh = focus * c.sensor_height_m / c.focal_length_m;
    {  // fitViewportToImageAspect (RayHelper.cpp:34-47)
        const double ia = W / H, va = vw / vh;
        if (ia > va) vh = vw / ia;
        else if (ia < va) vw = vh * ia;
    }
    const V3 w = normalize(V3(c.direction));
    V3 up(c.up);
    if (!finite_v(up) || len2(up) <= 1e-12) up = V3(0, 1, 0);
    up = normalize(up);
    if (len2(cross(up, w)) <= 1e-12) up = V3(0, 0, 1);
    if (len2(cross(up, w)) <= 1e-12) up = V3(1, 0, 0);
    const V3 u = normalize(cross(up, w));
    const V3 v = cross(w, u);
    const double aperture = c.pinhole ? 0.0 : c.focal_length_m / c.f_number;
    g.lens_radius = aperture / (2.0 * mpu);
    const V3 hz = u * vw, vt = v * vh;
    const V3 llc = pos + (hz / 2.0) + (vt / 2.0) + (w * focus);
    for (int a = 0; a < 3; a++) {
        g.position[a] = pos[a];
        g.u[a] = u[a];
        g.v[a] = v[a];
        g.horizontal[a] = hz[a];
        g.vertical[a] = vt[a];
        g.lower_left[a] = llc[a];
    }
    return g;
}

ScenePack* pack_scene(const LuzSceneDesc* d)
{
    if (!d) invalid("Scene description is NULL.");
    if (d->abi_version != LUZ_GPU_ABI_VERSION) invalid("Scene description ABI version mismatch.");
    if (d->material_count < 0 || d->object_count < 0 || d->mesh_count < 0 || d->texture_count < 0)
        invalid("Negative array size in scene description.");
    auto P = std::make_unique<ScenePack>();
    ScenePack& S = *P;
    GSceneConst& K = S.consts;
    S.camera = d->camera;
    {  // Camera setters (src/core/Camera.cpp) reject non-positive optics.
        const LuzCameraDesc& c = d->camera;
        if (!(c.focal_length_m > 0) || !std::isfinite(c.focal_length_m)) invalid("Camera focal length must be finite and positive.");
        if (!(c.sensor_width_m > 0) || !std::isfinite(c.sensor_width_m)) invalid("Camera sensor width must be finite and positive.");
        if (!(c.sensor_height_m > 0) || !std::isfinite(c.sensor_height_m)) invalid("Camera sensor height must be finite and positive.");
        if (!(c.f_number > 0) || !std::isfinite(c.f_number)) invalid("Camera f-number must be finite and positive.");
        if (!(c.focus_distance_m > 0) || !std::isfinite(c.focus_distance_m)) invalid("Camera focus distance must be finite and positive.");
    }
    if (!std::isfinite(d->meters_per_unit) || d->meters_per_unit <= 0.0)
        invalid("Scene meters per unit must be finite and positive.");
    K.meters_per_unit = d->meters_per_unit;

    // textures
    for (int i = 0; i < d->texture_count; i++) {
        const LuzTextureDesc& t = d->textures[i];
        if (t.width <= 0 || t.height <= 0 || !t.rgb) invalid("Texture dimensions must match the pixel count.");
        GTexture g{t.width, t.height, (int32_t)(S.texels.size() / 4), 0};
        for (int64_t k = 0; k < (int64_t)t.width * t.height; k++) {
            S.texels.push_back((float)t.rgb[3 * k]);
            S.texels.push_back((float)t.rgb[3 * k + 1]);
            S.texels.push_back((float)t.rgb[3 * k + 2]);
            S.texels.push_back(0.f);
        }
        S.textures.push_back(g);
    }
    for (int i = 0; i < d->material_count; i++) S.materials.push_back(pack_material(d->materials[i], d->texture_count));
    // IES profiles (IESProfile::load checks, IESProfile.cpp:186-223)
    if (d->ies_count < 0 || (d->ies_count > 0 && !d->ies)) invalid("IES profile list is inconsistent.");
    for (int i = 0; i < d->ies_count; i++) {
        const LuzIesDesc& q = d->ies[i];
        if (q.vertical_count <= 0) invalid("IES vertical angle count must be a positive integer.");
        if (q.horizontal_count <= 0) invalid("IES horizontal angle count must be a positive integer.");
        if (!q.vertical_deg || !q.horizontal_deg || !q.candela) invalid("IES profile has incomplete angle or candela data.");
        auto increasing = [&](const double* a, int n, const char* what) {
            for (int k = 0; k < n; k++) {
                if (!std::isfinite(a[k])) invalid(std::string(what) + " contain a non-finite value.");
                if (k > 0 && a[k] <= a[k - 1]) invalid(std::string(what) + " must be strictly increasing.");
            }
        };
        const int64_t nc = (int64_t)q.vertical_count * q.horizontal_count;
        for (int64_t k = 0; k < nc; k++)
            if (!std::isfinite(q.candela[k]) || q.candela[k] < 0.0)
                invalid("IES profile candela values must be finite and non-negative.");
        increasing(q.vertical_deg, q.vertical_count, "IES vertical angles");
        increasing(q.horizontal_deg, q.horizontal_count, "IES horizontal angles");
        const double flux = ies_flux(q.vertical_deg, q.vertical_count, q.horizontal_deg, q.horizontal_count, q.candela);
        if (!std::isfinite(flux) || flux <= 0.0) invalid("IES profile has zero luminous flux.");
        GIes g{q.vertical_count, q.horizontal_count, (int32_t)S.cdf.size(), 0, flux / (4.0 * kPi)};
        S.cdf.insert(S.cdf.end(), q.vertical_deg, q.vertical_deg + q.vertical_count);
        S.cdf.insert(S.cdf.end(), q.horizontal_deg, q.horizontal_deg + q.horizontal_count);
        S.cdf.insert(S.cdf.end(), q.candela, q.candela + nc);
        S.ies.push_back(g);
    }
    auto mat_type = [&](int m) {
        if (m < 0 || m >= d->material_count) invalid("Material index out of range.");
        return d->materials[m].type;
    };

    // meshes
    S.builds.resize(d->mesh_count);
    for (int mi = 0; mi < d->mesh_count; mi++) {
        const LuzMeshDesc& m = d->meshes[mi];
        mat_type(m.material);
        MeshBuild& mb = S.builds[mi];
        build_mesh(m, mb);
        if (mb.depth + 2 > kMeshStack)
            throw Status(LUZ_E_LIMIT, "Mesh BVH deeper than the traversal stack (128 entries).");
        S.max_mesh_depth = std::max(S.max_mesh_depth, mb.depth);
        GMesh g{};
        const std::size_t n = mb.area.size();
        g.tri_count = (int32_t)n;
        g.material = m.material;
        g.total_area = mb.total_area;
        g.depth = mb.depth;
        g.tri_offset = (int32_t)S.tris.size();
        g.node_offset = -1;
        g.normal_offset = -1;
        g.uv_offset = -1;
        if (n > 0) {
            put_box(mb.box, g.bmin, g.bmax);
            // interior nodes in preorder -> compact GNode indices
            std::vector<int32_t> gidx(mb.nodes.size(), -1);
            int32_t cnt = 0;
            for (std::size_t i = 0; i < mb.nodes.size(); i++)
                if (!mb.nodes[i].is_leaf) gidx[i] = cnt++;
            const int32_t base = (int32_t)S.nodes.size();
            S.nodes.reserve(S.nodes.size() + (std::size_t)cnt);
            S.nodes4.reserve(S.nodes4.size() + (std::size_t)cnt);
            S.tris.reserve(S.tris.size() + n);
            S.tri_shade.reserve(S.tri_shade.size() + n);
            S.cdf.reserve(S.cdf.size() + n);
            if (!mb.vn.empty()) S.vnormals.reserve(S.vnormals.size() + 9 * n);
            if (!mb.uv.empty()) S.vuvs.reserve(S.vuvs.size() + 6 * n);
            auto ref_of = [&](int64_t ni) -> uint32_t {
                const LuzMeshNode64& nd = mb.nodes[(std::size_t)ni];
                if (nd.is_leaf)
                    return kLeafBit | ((uint32_t)(g.tri_offset + nd.start) << 3) | (uint32_t)(nd.count - 1);
                return (uint32_t)(base + gidx[(std::size_t)ni]);
            };
            if ((uint64_t)(g.tri_offset + n) >= (1u << 28)) throw Status(LUZ_E_LIMIT, "Too many triangles (2^28).");
            for (std::size_t i = 0; i < mb.nodes.size(); i++) {
                const LuzMeshNode64& nd = mb.nodes[i];
                if (nd.is_leaf) continue;
                GNode gn{};
                Box64 lb, rb;
                const LuzMeshNode64& L = mb.nodes[(std::size_t)nd.left];
                const LuzMeshNode64& R = mb.nodes[(std::size_t)nd.right];
                for (int a = 0; a < 3; a++) {
                    lb.mn[a] = L.bmin[a];
                    lb.mx[a] = L.bmax[a];
                    rb.mn[a] = R.bmin[a];
                    rb.mx[a] = R.bmax[a];
                }
                put_box(lb, gn.lmin, gn.lmax);
                put_box(rb, gn.rmin, gn.rmax);
                gn.lref = ref_of(nd.left);
                gn.rref = ref_of(nd.right);
                S.nodes.push_back(gn);
            }
            g.node_offset = cnt > 0 ? base : -1;
            g.root_ref = (int32_t)ref_of(0);
            // Collapse every other level: one GNode4 per binary node N whose
            // children are visited together with it (preorder, parent first).
            g.node4_offset = -1;
            g.root4_ref = g.root_ref;
            if (cnt > 0) {
                g.node4_offset = (int32_t)S.nodes4.size();
                std::function<uint32_t(uint32_t)> collapse = [&](uint32_t bn) -> uint32_t {
                    const GNode b = S.nodes[bn];
                    const uint32_t qi = (uint32_t)S.nodes4.size();
                    S.nodes4.push_back(GNode4{});
                    GNode4 q{};
                    for (int a = 0; a < 3; a++) {
                        q.lmin[a] = b.lmin[a];
                        q.lmax[a] = b.lmax[a];
                        q.rmin[a] = b.rmin[a];
                        q.rmax[a] = b.rmax[a];
                    }
                    uint32_t sub[4] = {kEmptySlot, kEmptySlot, kEmptySlot, kEmptySlot};
                    for (int s = 0; s < 2; s++) {
                        const uint32_t c = s ? b.rref : b.lref;
                        const float* cmn = s ? b.rmin : b.lmin;
                        const float* cmx = s ? b.rmax : b.lmax;
                        if (c & kLeafBit) {
                            q.ref[2 * s] = c;
                            q.ref[2 * s + 1] = kEmptySlot;
                            for (int a = 0; a < 3; a++) {
                                q.cmin[2 * s][a] = cmn[a];
                                q.cmax[2 * s][a] = cmx[a];
                                q.cmin[2 * s + 1][a] = 0.f;
                                q.cmax[2 * s + 1][a] = 0.f;
                            }
                            continue;
                        }
                        const GNode cn = S.nodes[c];
                        for (int k = 0; k < 2; k++) {
                            const uint32_t gc = k ? cn.rref : cn.lref;
                            for (int a = 0; a < 3; a++) {
                                q.cmin[2 * s + k][a] = k ? cn.rmin[a] : cn.lmin[a];
                                q.cmax[2 * s + k][a] = k ? cn.rmax[a] : cn.lmax[a];
                            }
                            q.ref[2 * s + k] = gc;
                            if (!(gc & kLeafBit)) sub[2 * s + k] = gc;
                        }
                    }
                    for (int k = 0; k < 4; k++)
                        if (sub[k] != kEmptySlot) q.ref[k] = collapse(sub[k]);
                    S.nodes4[qi] = q;
                    return qi;
                };
                g.root4_ref = (int32_t)collapse((uint32_t)g.root_ref);
                // Relayout: the first kTopNodes4 nodes in breadth-first order, the rest in
                // the collapse's preorder. Only node indices move; every walk is unchanged.
                const uint32_t b = (uint32_t)g.node4_offset, e = (uint32_t)S.nodes4.size();
                std::vector<uint32_t> order{(uint32_t)g.root4_ref};
                for (std::size_t i = 0; i < order.size() && order.size() < (std::size_t)kTopNodes4; i++)
                    for (int k = 0; k < 4 && order.size() < (std::size_t)kTopNodes4; k++) {
                        const uint32_t r = S.nodes4[order[i]].ref[k];
                        if (!(r & kLeafBit)) order.push_back(r);
                    }
                std::vector<char> front(e - b, 0);
                for (uint32_t n : order) front[n - b] = 1;
                for (uint32_t n = b; n < e; n++)
                    if (!front[n - b]) order.push_back(n);
                std::vector<uint32_t> at(e - b);
                for (std::size_t i = 0; i < order.size(); i++) at[order[i] - b] = b + (uint32_t)i;
                std::vector<GNode4> re(e - b);
                for (std::size_t i = 0; i < order.size(); i++) {
                    GNode4 q = S.nodes4[order[i]];
                    for (int k = 0; k < 4; k++)
                        if (!(q.ref[k] & kLeafBit)) q.ref[k] = at[q.ref[k] - b];
                    re[i] = q;
                }
                std::copy(re.begin(), re.end(), S.nodes4.begin() + b);
                g.root4_ref = (int32_t)at[(uint32_t)g.root4_ref - b];
            }
            // triangles in leaf order
            const bool vn = !mb.vn.empty();
            const bool uv = !mb.uv.empty();
            if (vn) g.normal_offset = (int32_t)(S.vnormals.size() / 9);
            if (uv) g.uv_offset = (int32_t)(S.vuvs.size() / 6);
            g.slot_offset = (int32_t)S.index_pool.size();
            S.index_pool.resize(S.index_pool.size() + n);
            for (std::size_t slot = 0; slot < n; slot++) {
                const std::size_t t = (std::size_t)mb.order[slot];
                GTri tr{};
                for (int a = 0; a < 3; a++) {
                    tr.v0[a] = (float)mb.v0[3 * t + a];
                    tr.e1[a] = (float)mb.e1[3 * t + a];
                    tr.e2[a] = (float)mb.e2[3 * t + a];
                }
                tr.orig = (uint32_t)t;
                tr.area = (float)mb.area[t];
                S.tris.push_back(tr);
                GTriShade sh{};
                for (int a = 0; a < 3; a++) sh.fn[a] = (float)mb.fn[3 * t + a];
                sh.pad = (vn && mb.has_vn[t]) ? 1.f : 0.f;
                S.tri_shade.push_back(sh);
                if (vn)
                    for (int k = 0; k < 9; k++) S.vnormals.push_back((float)mb.vn[9 * t + k]);
                if (uv)
                    for (int k = 0; k < 6; k++) S.vuvs.push_back((float)mb.uv[6 * t + k]);
                S.index_pool[g.slot_offset + t] = g.tri_offset + (int32_t)slot;
            }
            // area prefix sums in original order (Mesh::_computePackedTriangleAreas)
            g.cdf_offset = (int32_t)S.cdf.size();
            double acc = 0.0;
            for (std::size_t t = 0; t < n; t++) {
                acc += mb.area[t];
                S.cdf.push_back(acc);
            }
        }
        S.meshes.push_back(g);
    }

    // objects
    struct Bounded {
        int obj;
        Box64 box;
    };
    std::vector<Bounded> bounded;
    std::vector<int32_t> unaccel;
    S.object_of_desc.assign(d->object_count, -1);
    std::vector<Box64> obj_box;
    bool scene_has_box = false;   // sceneBoundingBox (CausticPhotonMap.cpp:235-277): every box but directional lights'
    Box64 scene_box{};
    for (int i = 0; i < d->object_count; i++) {
        const LuzObjectDesc& o = d->objects[i];
        GObject g{};
        g.id = i;
        g.material = o.material;
        bool has_box = false, hittable = true;
        Box64 box{};
        switch (o.kind) {
        case LUZ_OBJ_RECTANGLE: {
            mat_type(o.material);
            RectBasis rb;
            g.kind = OK_RECT;
            if (o.has_uvs) {   // Rectangle::setTextureCoordinates: corners uv0..uv3 (x, y used)
                for (int c = 0; c < 4; c++) {
                    g.f[2 * c] = (float)o.uv[3 * c];
                    g.f[2 * c + 1] = (float)o.uv[3 * c + 1];
                }
                g.f[8] = 1.0f;
            }
            if (o.size[0] <= 0.0 || o.size[1] <= 0.0 || !rect_basis(o, rb)) {
                hittable = false;   // Rectangle::hit returns false; no bounding box
                g.aux = -1;
                break;
            }
            g.aux = (int32_t)S.rects.size();
            S.rects.push_back(make_rect(V3(o.position), rb, o.size[0], o.size[1]));
            has_box = rect_box(V3(o.position), rb, o.size[0], o.size[1], box);
            break;
        }
        case LUZ_OBJ_SPHERE: {
            mat_type(o.material);
            g.kind = OK_SPHERE;
            const double r = o.size[0];
            for (int a = 0; a < 3; a++) {
                g.f[a] = (float)o.position[a];
                box.mn[a] = o.position[a] - r;
                box.mx[a] = o.position[a] + r;
            }
            g.f[3] = (float)r;
            g.f[4] = o.visible ? 1.f : 0.f;
            if (o.uv_projection != 0 && o.uv_projection != 1) invalid("Unknown sphere UV projection.");
            g.f[5] = (float)o.uv_projection;
            has_box = true;
            if (o.ies != -1) {   // Sphere::setIESProfile (Sphere.cpp:188-202)
                if (o.ies < 0 || o.ies >= d->ies_count) invalid("IES profile index out of range.");
                const double l2 = o.ies_direction[0] * o.ies_direction[0] + o.ies_direction[1] * o.ies_direction[1]
                                + o.ies_direction[2] * o.ies_direction[2];
                if (!std::isfinite(l2) || l2 <= 0.0) invalid("IES profile direction must be non-zero.");
                if (!std::isfinite(o.ies_rotation_degrees)) invalid("IES profile rotation must be finite.");
            }
            break;
        }
        case LUZ_OBJ_CUBE: {
            mat_type(o.material);
            g.kind = OK_CUBE;
            g.aux = (int32_t)S.rects.size();
            const V3 p(o.position);
            const double W = o.size[0], Hh = o.size[1], D = o.size[2];
            struct Face {
                V3 c, n;
                double w, h;
            };
            // Cube::_generateFaces order (src/core/Hittables/Cube.cpp:80-101)
            const Face faces[6] = {
                {p - V3(0, 0, D / 2.0), V3(0, 0, -1), W, Hh}, {p + V3(0, 0, D / 2.0), V3(0, 0, 1), W, Hh},
                {p + V3(0, Hh / 2.0, 0), V3(0, 1, 0), W, D},   {p - V3(0, Hh / 2.0, 0), V3(0, -1, 0), W, D},
                {p + V3(W / 2.0, 0, 0), V3(1, 0, 0), D, Hh},   {p - V3(W / 2.0, 0, 0), V3(-1, 0, 0), D, Hh}};
            for (const Face& f : faces) {
                LuzObjectDesc fo{};
                fo.orientation[0] = f.n.x;
                fo.orientation[1] = f.n.y;
                fo.orientation[2] = f.n.z;
                RectBasis rb;
                rect_basis(fo, rb);
                S.rects.push_back(make_rect(f.c, rb, f.w, f.h));
            }
            for (int a = 0; a < 3; a++) {
                box.mn[a] = p[a] - o.size[a] / 2.0;
                box.mx[a] = p[a] + o.size[a] / 2.0;
            }
            has_box = true;
            break;
        }
        case LUZ_OBJ_PLANE: {
            mat_type(o.material);
            g.kind = OK_PLANE;
            g.f[0] = (float)o.position[1];
            for (int a = 0; a < 3; a++) g.f[1 + a] = (float)o.orientation[a];
            break;
        }
        case LUZ_OBJ_MESH: {
            if (o.mesh < 0 || o.mesh >= d->mesh_count) invalid("Mesh index out of range.");
            g.kind = OK_MESH;
            g.aux = o.mesh;
            g.material = d->meshes[o.mesh].material;
            if (S.builds[o.mesh].area.empty()) {
                hittable = false;
                break;
            }
            box = S.builds[o.mesh].box;
            has_box = true;
            break;
        }
        case LUZ_OBJ_MESH_INSTANCE: {
            if (o.mesh < 0 || o.mesh >= d->mesh_count) invalid("Mesh index out of range.");
            mat_type(o.material);
            g.kind = OK_INSTANCE;
            g.aux = o.mesh;
            const Xform x(o);
            for (int a = 0; a < 3; a++) {
                g.f[a] = (float)o.position[a];
                g.f[3 + a] = (float)o.scale[a];
            }
            g.f[6] = (float)x.cx;
            g.f[7] = (float)x.sx;
            g.f[8] = (float)x.cy;
            g.f[9] = (float)x.sy;
            g.f[10] = (float)x.cz;
            g.f[11] = (float)x.sz;
            const MeshBuild& mb = S.builds[o.mesh];
            if (mb.area.empty()) {
                hittable = false;
                break;
            }
            if (!x.invertible) hittable = false;   // _localRay fails; box still exists
            // MeshInstance::_computeBoundingBox (MeshInstance.cpp:193-243)
            const Box64& lb = mb.box;
            double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
            bool any = false;
            for (int c = 0; c < 8; c++) {
                const V3 corner((c & 1) ? lb.mx[0] : lb.mn[0], (c & 2) ? lb.mx[1] : lb.mn[1], (c & 4) ? lb.mx[2] : lb.mn[2]);
                const V3 wc = x.point(corner);
                if (!finite_v(wc)) continue;
                for (int a = 0; a < 3; a++) {
                    mn[a] = std::min(mn[a], wc[a]);
                    mx[a] = std::max(mx[a], wc[a]);
                }
                any = true;
            }
            if (any) {
                for (int a = 0; a < 3; a++) {
                    box.mn[a] = mn[a];
                    box.mx[a] = mx[a];
                }
                has_box = true;
            }
            break;
        }
        case LUZ_OBJ_VOLUME: {
            if (mat_type(o.material) == LUZ_MAT_EMISSIVE) unsupported("Emissive volume phase functions are not on the GPU path.");
            if (!std::isfinite(o.density) || o.density <= 0.0) invalid("Volume density must be finite and positive.");
            g.kind = OK_VOLUME;
            g.aux = o.boundary_kind;
            if (o.boundary_kind == LUZ_OBJ_CUBE) {
                for (int a = 0; a < 3; a++) {
                    box.mn[a] = o.position[a] - o.size[a] / 2.0;
                    box.mx[a] = o.position[a] + o.size[a] / 2.0;
                    g.f[a] = (float)box.mn[a];
                    g.f[3 + a] = (float)box.mx[a];
                }
            } else if (o.boundary_kind == LUZ_OBJ_SPHERE) {
                for (int a = 0; a < 3; a++) {
                    g.f[a] = (float)o.position[a];
                    box.mn[a] = o.position[a] - o.size[0];
                    box.mx[a] = o.position[a] + o.size[0];
                }
                g.f[3] = (float)o.size[0];
            } else {
                unsupported("Volume boundaries other than Cube and Sphere are not on the GPU path.");
            }
            g.f[6] = (float)(-1.0 / o.density);
            has_box = true;
            break;
        }
        case LUZ_OBJ_DIRECTIONAL_LIGHT: {
            mat_type(o.material);
            g.kind = OK_DIRECTIONAL;
            V3 dir(o.orientation);
            dir = len2(dir) <= 0.0 ? V3(0, -1, 0) : normalize(dir);
            put3(g.f, dir);
            hittable = false;   // DirectionalLight::hit always returns false
            break;
        }
        default:
            invalid("Unknown object kind " + std::to_string(o.kind) + ".");
        }
        const int32_t gi = (int32_t)S.objects.size();
        S.objects.push_back(g);
        obj_box.push_back(box);
        S.object_of_desc[i] = gi;
        if (has_box) {
            if (!scene_has_box) {
                scene_box = box;
                scene_has_box = true;
            } else {
                for (int a = 0; a < 3; a++) {
                    scene_box.mn[a] = std::min(scene_box.mn[a], box.mn[a]);
                    scene_box.mx[a] = std::max(scene_box.mx[a], box.mx[a]);
                }
            }
        }
        if (!hittable) continue;
        if (has_box) bounded.push_back({gi, box});
        else unaccel.push_back(gi);
    }

    // top level (Scene::updateAccelerationStructure)
    K.accel_kind = 0;
    K.accel_object = -1;
    if (bounded.size() == 1) {
        K.accel_kind = 2;
        K.accel_object = bounded[0].obj;
    } else if (bounded.size() > 1) {
        K.accel_kind = 1;
        std::vector<int> h(bounded.size());
        std::iota(h.begin(), h.end(), 0);
        struct TopTmp {
            std::vector<std::pair<bool, int>> kids;   // (is_node, index)
            Box64 box;
        };
        std::vector<TopTmp> tmp;
        std::function<int(std::size_t, std::size_t, bool)> rec = [&](std::size_t s, std::size_t e, bool root) -> int {
            const int me = (int)tmp.size();
            tmp.emplace_back();
            Box64 rb{};
            bool hb = false;
            for (std::size_t i = s; i < e; i++) {
                rb = hb ? merge_f(rb, bounded[h[i]].box) : bounded[h[i]].box;
                hb = true;
            }
            const int axis = largest_axis(rb);
            const std::size_t n = e - s;
            std::vector<std::pair<bool, int>> kids;
            if (n <= 8 || (root && n <= 16)) {
                for (std::size_t i = s; i < e; i++) kids.push_back({false, h[i]});
            } else {
                std::sort(h.begin() + s, h.begin() + e, [&](int a, int b) {
                    return bounded[a].box.mn[axis] < bounded[b].box.mn[axis];
                });
                const std::size_t mid = s + n / 2;
                const int l = rec(s, mid, false);
                const int r = rec(mid, e, false);
                kids.push_back({true, l});
                kids.push_back({true, r});
            }
            Box64 nb{};
            bool first = true;
            for (auto& k : kids) {
                const Box64& cb = k.first ? tmp[k.second].box : bounded[k.second].box;
                nb = first ? cb : merge_f(nb, cb);
                first = false;
            }
            tmp[me].kids = kids;
            tmp[me].box = nb;
            return me;
        };
        rec(0, bounded.size(), true);
        for (const TopTmp& t : tmp) {
            GTopNode n{};
            put_box(t.box, n.bmin, n.bmax);
            n.child_start = (int32_t)S.top_children.size();
            n.child_count = (int32_t)t.kids.size();
            for (auto& k : t.kids) {
                GTopChild c{};
                const Box64& cb = k.first ? tmp[k.second].box : bounded[k.second].box;
                put_box(cb, c.bmin, c.bmax);
                c.is_node = k.first ? 1 : 0;
                c.ref = k.first ? k.second : bounded[k.second].obj;
                S.top_children.push_back(c);
            }
            S.top_nodes.push_back(n);
        }
    }
    K.unaccel_offset = (int32_t)S.index_pool.size();
    K.unaccel_count = (int32_t)unaccel.size();
    for (int32_t u : unaccel) S.index_pool.push_back(u);

    // lights (Scene::updateLights) with their selection weights
    std::vector<double> weights;
    for (int i = 0; i < d->object_count; i++) {
        const LuzObjectDesc& o = d->objects[i];
        const GObject& g = S.objects[S.object_of_desc[i]];
        const int mat = g.material;
        if (mat < 0 || d->materials[mat].type != LUZ_MAT_EMISSIVE) continue;
        const double* em = d->materials[mat].color;
        const double lum = luminance(em);
        GLight L{};
        L.ies = -1;
        L.object = S.object_of_desc[i];
        L.material = mat;
        for (int a = 0; a < 3; a++) L.emitted[a] = (float)em[a];
        L.cdf_offset = -1;
        double w = 0.0;
        switch (o.kind) {
        case LUZ_OBJ_RECTANGLE: {
            L.kind = g.aux >= 0 ? LK_RECT : LK_NONE;
            const double area = o.size[0] * o.size[1];
            L.area = area;
            w = (area <= 0.0 || !std::isfinite(lum) || lum <= 0.0) ? 0.0 : area * lum;
            break;
        }
        case LUZ_OBJ_SPHERE: {
            L.kind = LK_SPHERE;
            L.ies = o.ies;
            for (int a = 0; a < 3; a++) L.ies_axis[a] = o.ies_direction[a];
            L.ies_rotation = o.ies_rotation_degrees;
            const double area = 4.0 * kPi * o.size[0] * o.size[0];
            L.area = area;
            w = (area <= 0.0 || !std::isfinite(lum) || lum <= 0.0) ? 0.0 : area * lum;
            break;
        }
        case LUZ_OBJ_MESH: {
            const MeshBuild& mb = S.builds[o.mesh];
            L.kind = mb.area.empty() ? LK_NONE : LK_MESH;
            L.mesh = o.mesh;
            L.area = mb.total_area;
            w = (mb.total_area <= 0.0 || !std::isfinite(lum) || lum <= 0.0) ? 0.0 : mb.total_area * lum;
            break;
        }
        case LUZ_OBJ_MESH_INSTANCE: {
            const MeshBuild& mb = S.builds[o.mesh];
            const Xform x(o);
            L.kind = (mb.area.empty() || !x.invertible) ? LK_NONE : LK_INSTANCE;
            L.mesh = o.mesh;
            L.uniform = x.uniform ? 1 : 0;
            double area = 0.0;
            if (x.uniform) {
                area = mb.total_area * x.uniform_scale;
            } else {
                // MeshInstance::_transformedAreaPrefixSums (MeshInstance.cpp:362-391)
                L.cdf_offset = (int32_t)S.cdf.size();
                double acc = 0.0;
                for (std::size_t t = 0; t < mb.area.size(); t++) {
                    const double* vt = &mb.vtx[9 * t];
                    const V3 w0 = x.point(V3(vt)), w1 = x.point(V3(vt + 3)), w2 = x.point(V3(vt + 6));
                    double ta = std::sqrt(len2(cross(w1 - w0, w2 - w0))) / 2.0;
                    if (!std::isfinite(ta) || ta <= 0.0) ta = 0.0;
                    acc += ta;
                    S.cdf.push_back(acc);
                }
                L.cdf_count = (int32_t)mb.area.size();
                area = acc;
                if (!std::isfinite(acc) || acc <= 0.0) L.cdf_count = 0;
            }
            if (!std::isfinite(area) || area <= 0.0) area = 0.0;
            L.area = area;
            w = (!std::isfinite(lum) || lum <= 0.0 || area <= 0.0) ? 0.0 : area * lum;
            break;
        }
        case LUZ_OBJ_DIRECTIONAL_LIGHT:
            L.kind = LK_DIRECTIONAL;
            w = (!std::isfinite(lum) || lum <= 0.0) ? 0.0 : lum;
            break;
        default:
            L.kind = LK_NONE;   // Hittable::sampleLight yields pdf 0; weight = luminance
            w = (!std::isfinite(lum) || lum <= 0.0) ? 0.0 : lum;
            break;
        }
        if (!std::isfinite(w) || w <= 0.0) w = 0.0;
        weights.push_back(w);
        S.lights.push_back(L);
    }
    K.light_count = (int32_t)S.lights.size();
    {
        double total = 0.0;
        std::vector<double> cum;
        for (double w : weights) {
            total += w;
            cum.push_back(total);
        }
        K.light_total_weight = total;
        K.light_cdf_offset = -1;
        if (total > 0.0 && !cum.empty()) {
            K.light_cdf_offset = (int32_t)S.cdf.size();
            S.cdf.insert(S.cdf.end(), cum.begin(), cum.end());
        }
    }

    for (int a = 0; a < 3; a++) {   // scene box for the radiance cache's position input
        const double ext = scene_has_box ? scene_box.mx[a] - scene_box.mn[a] : 0.0;
        K.box_lo[a] = scene_has_box ? (float)scene_box.mn[a] : 0.0f;
        K.box_inv[a] = (std::isfinite(ext) && ext > 0.0) ? (float)(1.0 / ext) : 1.0f;
    }

    // caustic photon map settings (Scene setters, Scene.cpp:317-360; CausticPhotonMap::build, :430-450)
    if (d->caustics.enabled) {
        const LuzCausticsDesc& c = d->caustics;
        if (c.photons < 0) invalid("Caustic photon count must be non-negative.");
        if (c.passes <= 0) invalid("Caustic pass count must be positive.");
        if (!std::isfinite(c.radius_meters) || c.radius_meters <= 0.0)
            invalid("Caustic radius must be finite and positive.");
        if (!std::isfinite(c.alpha) || c.alpha <= 0.0 || c.alpha > 1.0)
            invalid("Caustic alpha must be finite and in (0,1].");
        GCaustics& g = K.caustics;
        double radius = c.radius_meters;   // progressiveRadiusMeters (:356-368)
        for (int pass = 1; pass < c.passes; pass++)
            radius *= std::sqrt(((double)pass + c.alpha) / ((double)pass + 1.0));
        g.photons = c.photons;
        g.passes = c.passes;
        g.radius_m = radius;
        g.radius_su = radius / K.meters_per_unit;
        g.gather_area_m2 = M_PI * radius * radius;
        g.m2_per_area = K.meters_per_unit * K.meters_per_unit;
        g.enabled = (c.photons > 0 && !S.lights.empty() && radius > 0.0 && g.radius_su > 0.0 && g.gather_area_m2 > 0.0
                     && std::isfinite(g.radius_su)) ? 1 : 0;
        g.has_bounds = scene_has_box ? 1 : 0;
        if (scene_has_box) {   // sampleDirectionalEmission (:287-326)
            double diag2 = 0.0;
            for (int a = 0; a < 3; a++) {
                g.center[a] = (scene_box.mn[a] + scene_box.mx[a]) * 0.5;
                const double dd = scene_box.mx[a] - scene_box.mn[a];
                diag2 += dd * dd;
            }
            double r = std::sqrt(diag2) * 0.5;
            if (!std::isfinite(r) || r <= 0.0) r = 1.0;
            g.disk_radius = r + std::max(kTMin64, c.radius_meters / K.meters_per_unit);
        }
    }

    // sky / environment
    if (d->sky != LUZ_SKY_NONE && d->sky != LUZ_SKY_LINEAR && d->sky != LUZ_SKY_ATMOSPHERE && d->sky != LUZ_SKY_ENVIRONMENT)
        invalid("Unknown sky type.");
    K.sky = d->sky;
    if (d->sky == LUZ_SKY_ATMOSPHERE) {   // Atmosphere setters (Atmosphere.cpp:93-300)
        const LuzAtmosphereDesc& a = d->atmosphere;
        if (!std::isfinite(a.earth_radius) || a.earth_radius <= 0.0) invalid("Earth radius must be positive.");
        if (!std::isfinite(a.atmosphere_radius) || a.atmosphere_radius <= a.earth_radius)
            invalid("Atmosphere radius must be larger than Earth radius.");
        if (!std::isfinite(a.h_r) || a.h_r <= 0.0) invalid("Atmosphere HR must be positive.");
        if (!std::isfinite(a.h_m) || a.h_m <= 0.0) invalid("Atmosphere HM must be positive.");
        if (a.samples <= 0) invalid("Atmosphere sample count must be positive.");
        if (a.light_samples <= 0) invalid("Atmosphere light sample count must be positive.");
        if (!std::isfinite(a.stars_brightness) || a.stars_brightness < 0.0) invalid("Stars brightness must be non-negative.");
        const double l2 = a.sun_direction[0] * a.sun_direction[0] + a.sun_direction[1] * a.sun_direction[1]
                        + a.sun_direction[2] * a.sun_direction[2];
        if (!finite3(a.sun_direction) || l2 <= 0.0) invalid("Atmosphere sun direction must be finite and non-zero.");
        if (!finite3(a.sun_radiance) || a.sun_radiance[0] < 0.0 || a.sun_radiance[1] < 0.0 || a.sun_radiance[2] < 0.0)
            invalid("Atmosphere sun radiance must be finite and non-negative.");
        if (!std::isfinite(a.sun_radiance_scale) || a.sun_radiance_scale < 0.0)
            invalid("Atmosphere sun radiance scale must be finite and non-negative.");
        GAtmos& g = K.atmos;
        const double il = 1.0 / std::sqrt(l2);   // Utilities::normalize: (1 / length) * v
        for (int c = 0; c < 3; c++) {
            g.sun_dir[c] = il * a.sun_direction[c];
            g.sun_rad[c] = a.sun_radiance[c] * a.sun_radiance_scale;
        }
        g.earth_r = a.earth_radius;
        g.atmos_r = a.atmosphere_radius;
        g.inv_hr = 1.0 / a.h_r;
        g.inv_hm = 1.0 / a.h_m;
        g.stars = a.stars_brightness;
        g.samples = a.samples;
        g.light_samples = a.light_samples;
    }
    for (int a = 0; a < 3; a++) K.background[a] = (float)d->background[a];
    K.background_luminance = (float)luminance(d->background);
    GEnv& E = K.env;
    const LuzEnvironmentDesc& ed = d->environment;
    const bool has_map = ed.width > 0 && ed.height > 0 && ed.rgb;
    if (ed.width < 0 || ed.height < 0 || ((ed.width > 0) != (ed.height > 0)))
        invalid("Environment map dimensions must match the pixel count.");
    if (has_map) {
        E.width = ed.width;
        E.height = ed.height;
        E.strength = (float)ed.strength;
        E.rotation = ed.rotation_degrees;
        E.present = ed.strength > 0.0 ? 1 : 0;
        E.lighting = (ed.lighting && ed.strength > 0.0) ? 1 : 0;
        const int64_t WH = (int64_t)ed.width * ed.height;
        E.texel_offset = 0;
        S.env_texels.resize(4 * WH);
        for (int64_t k = 0; k < WH; k++) {
            S.env_texels[4 * k] = (float)ed.rgb[3 * k];
            S.env_texels[4 * k + 1] = (float)ed.rgb[3 * k + 1];
            S.env_texels[4 * k + 2] = (float)ed.rgb[3 * k + 2];
        }
        // EnvironmentMap::buildDistribution (src/core/EnvironmentMap.cpp:627-671)
        std::vector<double> w(WH), sa(WH), cdf;
        cdf.reserve(WH);
        double total = 0.0;
        const double dphi = 2.0 * kPi / (double)ed.width;
        for (int y = 0; y < ed.height; y++) {
            const double t0 = kPi * (double)y / (double)ed.height;
            const double t1 = kPi * (double)(y + 1) / (double)ed.height;
            const double s = dphi * std::max(0.0, std::cos(t0) - std::cos(t1));
            for (int x = 0; x < ed.width; x++) {
                const int64_t k = (int64_t)y * ed.width + x;
                double c[3];
                for (int a = 0; a < 3; a++) {
                    const double v = ed.rgb[3 * k + a];
                    c[a] = std::isfinite(v) ? std::max(0.0, v) : 0.0;
                }
                const double lum = luminance(c);
                const double wt = (std::isfinite(lum) && lum > 0.0) ? lum * s : 0.0;
                sa[k] = s;
                w[k] = wt;
                total += wt;
                cdf.push_back(total);
            }
        }
        if (!std::isfinite(total) || total <= 0.0) {
            total = 0.0;
            cdf.clear();
        }
        E.total_weight = total;
        E.cdf_offset = (int64_t)S.cdf.size();
        E.guide_offset = -1;
        if (total > 0.0) {
            // Guide tables for the device-side std::lower_bound. For bucket b of K:
            //   lo[b] = first index with cdf >= (b/K) total (1 - eps)
            //   hi[b] = first index with cdf >= ((b+1)/K) total (1 + eps), plus one
            // so for any target whose computed bucket is b (even if rounding moved
            // it across a bucket edge) the lower_bound answer lies in [lo[b], hi[b]).
            const int32_t K = (int32_t)std::min<int64_t>(65536, std::max<int64_t>(1, WH / 4));
            const double eps = 1e-9;
            E.guide_count = K;
            E.guide_offset = (int32_t)S.index_pool.size();
            auto first_ge = [&](double thr) {
                return (int64_t)(std::lower_bound(cdf.begin(), cdf.end(), thr) - cdf.begin());
            };
            for (int32_t b = 0; b < K; b++)
                S.index_pool.push_back((int32_t)std::min<int64_t>(first_ge(((double)b / K) * total * (1.0 - eps)), WH - 1));
            for (int32_t b = 0; b < K; b++)
                S.index_pool.push_back((int32_t)std::min<int64_t>(first_ge(((double)(b + 1) / K) * total * (1.0 + eps)) + 1, WH));
            S.cdf.insert(S.cdf.end(), cdf.begin(), cdf.end());
            E.pdf_offset = (int64_t)S.cdf.size();
            for (int64_t k = 0; k < WH; k++)
                S.cdf.push_back((w[k] <= 0.0 || sa[k] <= 0.0) ? 0.0 : ((w[k] / total) / sa[k]));
        } else {
            E.pdf_offset = -1;
        }
    }
    // Shade binning: the material type (1..7) a hit on each object shades with
    // (make_hit: a mesh shades with its mesh's material, every other kind with its own).
    S.obj_class.assign(S.objects.size(), 0);
    for (std::size_t i = 0; i < S.objects.size(); i++) {
        const GObject& o = S.objects[i];
        const int32_t mat = o.kind == OK_MESH ? S.meshes[(std::size_t)o.aux].material : o.material;
        if (mat >= 0 && (std::size_t)mat < S.materials.size()) S.obj_class[i] = (uint8_t)S.materials[(std::size_t)mat].type;
    }
    // Traversal kernel specialisation (TraceFeature bits: 1 instances, 2 volumes).
    K.features = 0;
    K.cube_cross_spheres = 0;
    for (const GObject& o : S.objects) {
        if (o.kind == OK_INSTANCE) K.features |= 1;
        if (o.kind == OK_VOLUME) K.features |= 2;
        if (o.kind == OK_SPHERE && o.f[5] != 0.f) K.cube_cross_spheres = 1;
    }
    const double bg_max = std::max(d->background[0], std::max(d->background[1], d->background[2]));
    K.has_constant_background_light = (!E.lighting && d->sky == LUZ_SKY_NONE && bg_max > 0.0) ? 1 : 0;
    K.sampled_infinite_light = (E.lighting || K.has_constant_background_light) ? 1 : 0;
    return P.release();
}

}  // namespace luz
