// geometry.cu -- host-side beam geometry and library bookkeeping.
//
// The beam geometry (calc_range, canonical beamlets) runs once per plan on the
// host in single precision with the reference's operation order, because the
// reference computes it that way on the CPU and every downstream index (long_dim,
// BEV depth offsets) must come out identical: BEAM_h::calc_range
// (FastDoseLib/src/beam.cu:134-222) and IMRT::BeamBundle::beamletInit
// (IMRTOpt/src/IMRTBeamBundle.cu:341-569).
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "fd2_internal.cuh"

namespace fd2 {

static thread_local char g_last_error[512] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

namespace {

constexpr float kEps = 1e-4f;  // eps_fastdose (FastDoseLib/include/macros.h:21)
constexpr float kPi = 3.14159265358979323846f;

struct V3 {
    float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float len(V3 a) { return std::sqrt(dot(a, a)); }
// 1/sqrt(x) rounded once from the exact value; equal to what the reference's
// host normalize() returns for every input we compared.
inline float rsqrt_cr(float x) { return (float)(1.0 / std::sqrt((double)x)); }
inline V3 normalize(V3 a) { return a * rsqrt_cr(dot(a, a)); }
inline float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// Rodrigues rotation of p about the unit axis r by t.
V3 rotate_axis(V3 p, V3 r, float t) {
    float s = std::sin(t), c = std::cos(t);
    float k = (1.0f - c) * (p.x * r.x + p.y * r.y + p.z * r.z);
    return v3(k * r.x + c * p.x + s * (r.y * p.z - r.z * p.y), k * r.y + c * p.y + s * (r.z * p.x - r.x * p.z),
              k * r.z + c * p.z + s * (r.x * p.y - r.y * p.x));
}

// BEV -> PVCS: undo collimator(+couch correction) about y, then gantry about the couch axis.
V3 bev_to_pvcs(V3 v, float th, float ph, float co) {
    V3 t = rotate_axis(v, v3(0, 1, 0), -(ph + co));
    return rotate_axis(t, v3(std::sin(-ph), 0, std::cos(-ph)), th);
}

}  // namespace

int calc_range(fd2_beam_t* b, const fd2_volume_t* vol) {
    float hx = b->fmap_size[0] * b->beamlet_size[0] / 2;
    float hy = b->fmap_size[1] * b->beamlet_size[1] / 2;
    // the fifth ray is the central axis; corner 2 keeps the reference's use of
    // the x half-size for its z component
    V3 rays[5] = {v3(hx, b->sad, hy), v3(hx, b->sad, -hy), v3(-hx, b->sad, hx), v3(-hx, b->sad, -hy),
                  v3(0, b->sad, 0)};
    for (auto& r : rays) r = bev_to_pvcs(r, b->angles[0], b->angles[1], b->angles[2]);
    V3 src = bev_to_pvcs(v3(0, -b->sad, 0), b->angles[0], b->angles[1], b->angles[2]) +
             v3(b->isocenter[0], b->isocenter[1], b->isocenter[2]);
    b->source[0] = src.x; b->source[1] = src.y; b->source[2] = src.z;
    V3 lo = v3(vol->bbox_start[0] * vol->voxel_size[0], vol->bbox_start[1] * vol->voxel_size[1],
               vol->bbox_start[2] * vol->voxel_size[2]);
    V3 hi = v3((vol->bbox_start[0] + vol->bbox_dim[0]) * vol->voxel_size[0],
               (vol->bbox_start[1] + vol->bbox_dim[1]) * vol->voxel_size[1],
               (vol->bbox_start[2] + vol->bbox_dim[2]) * vol->voxel_size[2]);
    float dmin = 3.402823466e+38f, dmax = 1.175494351e-38f;
    bool hit = false;
    for (const V3& r : rays) {
        V3 pts[6];
        for (int j = 0; j < 3; j++) {
            double den = comp(r, j);
            den = std::signbit(den) ? den - kEps : den + kEps;
            double a1 = (comp(lo, j) - comp(src, j)) / den;
            double a2 = (comp(hi, j) - comp(src, j)) / den;
            pts[2 * j] = src + r * (float)a1;
            pts[2 * j + 1] = src + r * (float)a2;
        }
        for (int j = 0; j < 3; j++) {
            int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            for (int k = 0; k < 2; k++) {
                V3 p = pts[2 * j + k];
                if (comp(p, j1) >= comp(lo, j1) && comp(p, j1) <= comp(hi, j1) && comp(p, j2) >= comp(lo, j2) &&
                    comp(p, j2) <= comp(hi, j2)) {
                    float l = len(p - src) * b->sad / len(r);  // depth along the central axis
                    dmin = std::fmin(l, dmin);
                    dmax = std::fmax(l, dmax);
                    hit = true;
                }
            }
        }
    }
    FD2_REQUIRE(hit, FD2_ERR_GEOMETRY, "beam does not intersect the bounding box");
    b->lim_min = dmin;
    b->lim_max = dmax;
    b->long_dim = (uint32_t)std::ceil((b->lim_max - b->lim_min) / b->long_spacing);
    return FD2_OK;
}

int beamlet_init(const fd2_bundle_t* bb, int ix, int iy, const fd2_volume_t* vol, fd2_beam_t* out) {
    FD2_REQUIRE(bb && vol && out, FD2_ERR_INVALID_ARGUMENT, "beamlet_init: null argument");
    FD2_REQUIRE(ix >= 0 && iy >= 0 && ix < bb->fluence_dim[0] && iy < bb->fluence_dim[1], FD2_ERR_INVALID_ARGUMENT,
                "beamlet_init: pixel (%d, %d) outside the fluence map", ix, iy);
    const float bx = bb->beamlet_size[0], by = bb->beamlet_size[1];
    const float hfx = bb->fluence_dim[0] * bx * 0.5f, hfy = bb->fluence_dim[1] * by * 0.5f;
    // unit vectors from the source to the four corners of the pixel at the SAD plane
    V3 c[4] = {normalize(v3(ix * bx - hfx, bb->sad, iy * by - hfy)),
               normalize(v3((ix + 1) * bx - hfx, bb->sad, iy * by - hfy)),
               normalize(v3((ix + 1) * bx - hfx, bb->sad, (iy + 1) * by - hfy)),
               normalize(v3(ix * bx - hfx, bb->sad, (iy + 1) * by - hfy))};
    // Candidate axes: the bisector of either diagonal.  The corners are projected
    // onto the plane through the axis tip; the inscribed canonical (equal-edge)
    // pyramid's half-diagonal is the smallest corner distance (excluding the
    // diagonal's far corner).
    V3 axis[2], proj[2][4];
    float dist[2];
    for (int cs = 0; cs < 2; cs++) {
        V3 l = normalize(cs == 0 ? c[0] + c[2] : c[1] + c[3]);
        axis[cs] = l;
        float d[4];
        for (int q = 0; q < 4; q++) {
            proj[cs][q] = c[q] / dot(c[q], l);
            d[q] = len(proj[cs][q] - l);
        }
        if (cs == 0) {
            FD2_REQUIRE(std::fabs(d[0] - d[2]) <= kEps, FD2_ERR_GEOMETRY, "beamlet_init: asymmetric diagonal");
            dist[0] = std::fmin(std::fmin(d[0], d[1]), d[3]);
        } else {
            FD2_REQUIRE(std::fabs(d[1] - d[3]) <= kEps, FD2_ERR_GEOMETRY, "beamlet_init: asymmetric diagonal");
            dist[1] = std::fmin(std::fmin(d[0], d[1]), d[2]);
        }
    }
    const int cs = dist[0] > dist[1] ? 0 : 1;
    const V3 dir = axis[cs];
    V3 e0 = normalize(proj[cs][0] - dir), e1 = normalize(proj[cs][1] - dir);
    // the first case sums e0 with itself, as the reference does
    V3 codir = normalize(cs == 0 ? e0 + e0 : e0 + e1);
    float sad_r = bb->sad / dir.y;
    float fl_h = len((e0 + e1) * dist[cs] * 0.5f) * sad_r * 2;
    float fl_w = len((e0 - e1) * dist[cs] * 0.5f) * sad_r * 2;

    // gantry/couch of the beamlet axis: four sign cases tried in the reference's order
    V3 dpv = bev_to_pvcs(dir, bb->angles[0], bb->angles[1], bb->angles[2]);
    const V3 yax = v3(0, 1, 0);
    float theta = std::acos(dot(dpv, yax));
    float phi = std::asin(dpv.z * rsqrt_cr(dpv.z * dpv.z + dpv.x * dpv.x + kEps * kEps));
    const float ct[4] = {theta, theta, -theta, -theta};
    const float cp[4] = {phi, kPi - phi, phi, kPi - phi};
    int found = -1;
    for (int q = 0; q < 4 && found < 0; q++)
        if (!(dot(bev_to_pvcs(yax, ct[q], cp[q], 0.0f), dpv) < 1 - kEps)) found = q;
    FD2_REQUIRE(found >= 0, FD2_ERR_GEOMETRY, "beamlet_init: gantry/couch fit failed");
    const float th = ct[found], ph = cp[found];

    // collimator from the co-direction, two sign cases
    V3 cdpv = bev_to_pvcs(codir, bb->angles[0], bb->angles[1], bb->angles[2]);
    const V3 cbev = v3(0, 0, -1);
    float cosc = dot(cdpv, bev_to_pvcs(cbev, th, ph, 0.0f));
    cosc = cosc < -1.0f ? -1.0f : (cosc > 1.0f ? 1.0f : cosc);
    float coll = std::acos(cosc);
    if (dot(bev_to_pvcs(cbev, th, ph, coll), cdpv) < 1 - kEps * 10) {
        coll = -coll;
        FD2_REQUIRE(!(dot(bev_to_pvcs(cbev, th, ph, coll), cdpv) < 1 - kEps * 10), FD2_ERR_GEOMETRY,
                    "beamlet_init: collimator fit failed");
    }

    std::memset(out, 0, sizeof(*out));
    out->angles[0] = th; out->angles[1] = ph; out->angles[2] = coll;
    V3 disp = bev_to_pvcs(v3((ix + 0.5f - 0.5f * bb->fluence_dim[0]) * bx, 0.0f,
                             (iy + 0.5f - 0.5f * bb->fluence_dim[1]) * by),
                          bb->angles[0], bb->angles[1], bb->angles[2]);
    out->isocenter[0] = bb->isocenter[0] + disp.x;
    out->isocenter[1] = bb->isocenter[1] + disp.y;
    out->isocenter[2] = bb->isocenter[2] + disp.z;
    out->beamlet_size[0] = fl_w / bb->sub_fluence_on[0];
    out->beamlet_size[1] = fl_h / bb->sub_fluence_on[1];
    out->fmap_size[0] = (uint32_t)bb->sub_fluence_dim[0];
    out->fmap_size[1] = (uint32_t)bb->sub_fluence_dim[1];
    out->sad = sad_r;
    out->long_spacing = bb->long_spacing;
    uint64_t pitch = (uint64_t)out->fmap_size[0] * out->fmap_size[1] * sizeof(float);
    out->TermaBEV_pitch = pitch;
    out->DensityBEV_pitch = pitch;
    return calc_range(out, vol);
}

void cone_direction(const fd2_beam_t& b, float theta, float phi, float out[3]) {
    double st = std::sin((double)theta), ct = std::cos((double)theta);
    double sp = std::sin((double)phi), cp = std::cos((double)phi);
    double v[3] = {st * cp / b.beamlet_size[0], st * sp / b.beamlet_size[1], ct / b.long_spacing};
    double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int i = 0; i < 3; i++) out[i] = (float)(v[i] / n);
}

}  // namespace fd2

extern "C" {

const char* fd2_status_string(int s) {
    switch (s) {
        case FD2_OK: return "ok";
        case FD2_ERR_INVALID_ARGUMENT: return "invalid argument";
        case FD2_ERR_CUDA: return "CUDA error";
        case FD2_ERR_OUT_OF_MEMORY: return "out of device memory";
        case FD2_ERR_IO: return "I/O error";
        case FD2_ERR_GEOMETRY: return "geometry error";
        case FD2_ERR_CAPACITY: return "buffer too small";
        case FD2_ERR_WATCHDOG: return "device loop iteration cap reached";
        case FD2_ERR_NOT_SUPPORTED: return "not supported";
        case FD2_ERR_ADMISSION: return "request exceeds the admission budget";
        default: return "unknown status";
    }
}

int fd2_version(void) { return 100; }

const char* fd2_last_error(void) { return fd2::g_last_error; }

int fd2_beam_calc_range(fd2_beam_t* beam, const fd2_volume_t* volume) {
    FD2_REQUIRE(beam && volume, FD2_ERR_INVALID_ARGUMENT, "calc_range: null argument");
    return fd2::calc_range(beam, volume);
}

int fd2_beamlet_init(const fd2_bundle_t* bundle, int ix, int iy, const fd2_volume_t* volume, fd2_beam_t* out) {
    return fd2::beamlet_init(bundle, ix, iy, volume, out);
}

int fd2_bundles_beamlets(size_t n_bundles, const fd2_bundle_t* bundles, const uint8_t* flags,
                         const fd2_volume_t* volume, int n_threads, size_t cap, fd2_beam_t* out, uint32_t* counts) {
    FD2_REQUIRE((n_bundles == 0 || (bundles && flags && counts)) && volume && (cap == 0 || out),
                FD2_ERR_INVALID_ARGUMENT, "bundles_beamlets: null argument");
    // flagged pixels of each bundle, their flag offsets and output offsets
    std::vector<size_t> foff(n_bundles + 1, 0), boff(n_bundles + 1, 0);
    for (size_t b = 0; b < n_bundles; b++) {
        const int fx = bundles[b].fluence_dim[0], fy = bundles[b].fluence_dim[1];
        FD2_REQUIRE(fx > 0 && fy > 0, FD2_ERR_INVALID_ARGUMENT, "bundles_beamlets: bundle %zu has no fluence map", b);
        foff[b + 1] = foff[b] + (size_t)fx * fy;
        size_t c = 0;
        for (size_t k = foff[b]; k < foff[b + 1]; k++) c += flags[k] != 0;
        counts[b] = (uint32_t)c;
        boff[b + 1] = boff[b] + c;
    }
    FD2_REQUIRE(boff[n_bundles] <= cap, FD2_ERR_CAPACITY, "bundles_beamlets: %zu beamlets, room for %zu",
                boff[n_bundles], cap);
    int threads = n_threads > 0 ? n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    threads = (int)std::min<size_t>((size_t)threads, std::max<size_t>(n_bundles, 1));
    std::mutex mu;
    int first_rc = FD2_OK;
    std::string first_msg;
    auto work = [&](int t) {
        for (size_t b = (size_t)t; b < n_bundles; b += (size_t)threads) {
            const int fx = bundles[b].fluence_dim[0], fy = bundles[b].fluence_dim[1];
            size_t o = boff[b];
            for (int iy = 0; iy < fy; iy++)
                for (int ix = 0; ix < fx; ix++) {
                    if (!flags[foff[b] + (size_t)iy * fx + ix]) continue;
                    const int rc = fd2::beamlet_init(&bundles[b], ix, iy, volume, &out[o++]);
                    if (rc) {
                        std::lock_guard<std::mutex> lock(mu);
                        if (!first_rc) {
                            first_rc = rc;
                            first_msg = fd2_last_error();
                        }
                        return;
                    }
                }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    if (first_rc) fd2::set_error("%s", first_msg.c_str());
    return first_rc;
}

int fd2_beamlet_fluence(const fd2_bundle_t* bb, float* out, size_t n) {
    FD2_REQUIRE(bb && out, FD2_ERR_INVALID_ARGUMENT, "beamlet_fluence: null argument");
    int fx = bb->sub_fluence_dim[0], fy = bb->sub_fluence_dim[1];
    FD2_REQUIRE(n >= (size_t)fx * fy, FD2_ERR_CAPACITY, "beamlet_fluence: need %d floats", fx * fy);
    std::memset(out, 0, sizeof(float) * fx * fy);
    // centred open square (IMRTOpt/src/IMRTBeamBundle.cu:553-563)
    int lx = (int)((fx - bb->sub_fluence_on[0]) * 0.5f), ly = (int)((fy - bb->sub_fluence_on[1]) * 0.5f);
    for (int j = ly; j < ly + bb->sub_fluence_on[1]; j++)
        for (int i = lx; i < lx + bb->sub_fluence_on[0]; i++) out[i + j * fx] = 1.0f;
    return FD2_OK;
}

}  // extern "C"
