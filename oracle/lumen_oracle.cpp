/*
 * lumen_oracle.cpp - CPU oracle for the forward splatting path.
 *
 * TEST INFRASTRUCTURE ONLY: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, as the checker and as the
 * timed CPU baseline. The product (lumen_b200/) never links or calls it.
 *
 * A literal restatement of the reference Mojo path, same operation order,
 * same guards, same truncations; compiled with -ffp-contract=off so no
 * multiply-add is fused. Each function cites the Mojo lines it restates
 * (paths relative to the reference project root).
 *
 *   rasterize_scene            src/raster/pipeline.mojo:48-231
 *   Gaussian3D / get_gaussian  src/scene/gaussian.mojo:27-37,109-114
 *   PinholeCamera              src/scene/camera.mojo:24-40,66-79
 *   Quatf                      src/math/quaternion.mojo:46-117
 *   Vec3f.normalized           src/math/vector.mojo:100-110
 *   Covariance3D               src/math/covariance.mojo:41-83
 *   EWA / Jacobian / inverse   src/math/projection.mojo:10-148
 *   solve_eigenvalues_2x2      src/math/cholesky.mojo:28-51
 *   FrustumCuller              src/raster/culling.mojo:35-71
 *   TileGrid                   src/raster/tile.mojo:20-97
 *   SH basis and colour        src/math/spherical_harmonics.mojo:17-172
 *   keys and radix sort        src/raster/radix_sort.mojo:8-87
 *   TileRangeIndex             src/raster/binning.mojo:10-73
 *   compositor                 src/raster/compositor.mojo:10-89
 *   constants                  src/core/types.mojo:21-36
 *   compute_l1_loss            src/optim/loss.mojo:11-35
 *
 * Parity is pinned by the reference's known-answer tests (restated in
 * tests/test_oracle_kat.py); the Mojo code itself cannot run here.
 * The float32 exponential is lumen_expf (lumen_b200/csrc/lumen_expf.h), the
 * one function shared with the CUDA kernels, because Mojo's exp cannot be
 * observed and alpha-threshold decisions must agree bit for bit.
 *
 * Literal constants are written (T)(double literal): the reference's
 * FloatLiteral values are materialised as Float32 from a 64-bit literal.
 *
 * Float-to-Int conversion (Mojo Int(x) on a Float32): truncation toward zero;
 * for NaN or magnitudes >= 2^63 the reference's x86-64 conversion yields
 * INT64_MIN, restated by mojo_int().
 */
#include "lumen_oracle.h"
#include "../lumen_b200/csrc/lumen_expf.h"

#include <cmath>
#include <cstring>
#include <cstdint>
#include <vector>
#include <algorithm>
#include <thread>
#include <atomic>

namespace {

/* Static split of [0, n) over nt threads: f(lo, hi, thread_index). */
template <class F> static void parallel_for(int64_t n, int nt, F f) {
    if (nt <= 1 || n < 2) { f(0, n, 0); return; }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; ++t) th.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt, t); });
    for (auto& x : th) x.join();
}

/* Dynamic split of [0, n) in chunks: f(i). */
template <class F> static void parallel_dynamic(int64_t n, int nt, int64_t chunk, F f) {
    if (nt <= 1) { for (int64_t i = 0; i < n; ++i) f(i); return; }
    std::atomic<int64_t> next(0);
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&] {
            for (;;) {
                int64_t lo = next.fetch_add(chunk);
                if (lo >= n) break;
                int64_t hi = std::min(n, lo + chunk);
                for (int64_t i = lo; i < hi; ++i) f(i);
            }
        });
    for (auto& x : th) x.join();
}

template <typename T> struct Num;
template <> struct Num<float> {
    static float exp(float x) { return lumen_expf(x); }
};
template <> struct Num<double> {
    static double exp(double x) { return std::exp(x); }
};

template <typename T> static inline int64_t mojo_int(T x) {
    if (!(x > T(-9.2233720368547758e18) && x < T(9.2233720368547758e18))) return INT64_MIN;
    return (int64_t)x;
}

/* ---- constants, src/core/types.mojo:21-36 ---- */
template <typename T> struct K {
    static T min_alpha() { return (T)0.00392156862; }  /* MIN_ALPHA_THRESHOLD */
    static T t_eps() { return (T)0.0001; }              /* TRANSMITTANCE_EPSILON */
};

/* ---- Vec3f, src/math/vector.mojo:55-116 ---- */
template <typename T> struct V3 {
    T x, y, z;
    V3 sub(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    T length() const { return std::sqrt(x * x + y * y + z * z); }
    V3 normalized() const {                      /* vector.mojo:106-110 */
        T l = length();
        if (l > (T)0.000001) return {x / l, y / l, z / l};
        return {T(0), T(0), T(0)};
    }
};

/* ---- Mat3x3f, src/math/matrix.mojo:62-98 ---- */
template <typename T> struct M3 { T m00, m01, m02, m10, m11, m12, m20, m21, m22; };

/* ---- Quatf, src/math/quaternion.mojo:9-117 ---- */
template <typename T> struct Q {
    T w, x, y, z;
    static Q identity() { return {T(1), T(0), T(0), T(0)}; }
    T norm_squared() const { return w * w + x * x + y * y + z * z; }   /* :46-47 */
    Q normalized() const {                                             /* :52-57 */
        T n = std::sqrt(norm_squared());
        if (n > (T)0.000001) {
            T inv_n = T(1) / n;
            return {w * inv_n, x * inv_n, y * inv_n, z * inv_n};
        }
        return identity();
    }
    Q inverse() const {                                                /* :62-67 */
        T ns = norm_squared();
        if (ns > (T)0.000001) {
            T inv_ns = T(1) / ns;
            return {w * inv_ns, -x * inv_ns, -y * inv_ns, -z * inv_ns};
        }
        return identity();
    }
    Q mul(const Q& o) const {                                          /* :69-78 */
        return {w * o.w - x * o.x - y * o.y - z * o.z,
                w * o.x + x * o.w + y * o.z - z * o.y,
                w * o.y - x * o.z + y * o.w + z * o.x,
                w * o.z + x * o.y - y * o.x + z * o.w};
    }
    V3<T> rotate_vec(const V3<T>& v) const {                           /* :80-87 */
        Q p{T(0), v.x, v.y, v.z};
        Q q_inv = inverse();
        Q r = mul(p).mul(q_inv);
        return {r.x, r.y, r.z};
    }
    M3<T> to_rotation_matrix() const {                                 /* :89-117 */
        Q q = normalized();
        T w_ = q.w, x_ = q.x, y_ = q.y, z_ = q.z;
        T x2 = x_ + x_, y2 = y_ + y_, z2 = z_ + z_;
        T xx = x_ * x2, xy = x_ * y2, xz = x_ * z2;
        T yy = y_ * y2, yz = y_ * z2, zz = z_ * z2;
        T wx = w_ * x2, wy = w_ * y2, wz = w_ * z2;
        return {T(1) - (yy + zz), xy - wz, xz + wy,
                xy + wz, T(1) - (xx + zz), yz - wx,
                xz - wy, yz + wx, T(1) - (xx + yy)};
    }
};

/* ---- PinholeCamera, src/scene/camera.mojo:24-79 ---- */
template <typename T> struct Cam {
    V3<T> position;
    Q<T> rotation;
    T fx, fy, cx, cy, near_plane, far_plane;
    int64_t width, height;
    explicit Cam(const OracleCamera& c) {
        position = {T(c.position[0]), T(c.position[1]), T(c.position[2])};
        Q<T> r{T(c.rotation[0]), T(c.rotation[1]), T(c.rotation[2]), T(c.rotation[3])};
        rotation = r.normalized();                                     /* :229 */
        fx = T(c.fx); fy = T(c.fy); cx = T(c.cx); cy = T(c.cy);
        near_plane = T(c.near_plane); far_plane = T(c.far_plane);
        width = c.width; height = c.height;
    }
    M3<T> view_rotation() const { return rotation.inverse().to_rotation_matrix(); } /* :66-67 */
    V3<T> world_to_cam(const V3<T>& p) const {                         /* :69-71 */
        V3<T> rel = p.sub(position);
        return rotation.inverse().rotate_vec(rel);
    }
    void cam_to_screen(const V3<T>& p, T& u, T& v) const {             /* :73-79 */
        T tz = p.z;
        if (tz < (T)0.0001 && tz > (T)-0.0001) tz = (T)0.0001;
        u = fx * (p.x / tz) + cx;
        v = fy * (p.y / tz) + cy;
    }
};

/* ---- Covariance3D.from_scale_and_rotation, src/math/covariance.mojo:41-83 ---- */
template <typename T> static void cov3d(const V3<T>& s, const Q<T>& rot, T c[6]) {
    T sx = s.x; if (sx < (T)0.00001) sx = (T)0.00001;
    T sy = s.y; if (sy < (T)0.00001) sy = (T)0.00001;
    T sz = s.z; if (sz < (T)0.00001) sz = (T)0.00001;
    M3<T> R = rot.to_rotation_matrix();
    T m00 = R.m00 * sx, m01 = R.m01 * sy, m02 = R.m02 * sz;
    T m10 = R.m10 * sx, m11 = R.m11 * sy, m12 = R.m12 * sz;
    T m20 = R.m20 * sx, m21 = R.m21 * sy, m22 = R.m22 * sz;
    c[0] = m00 * m00 + m01 * m01 + m02 * m02;
    c[1] = m00 * m10 + m01 * m11 + m02 * m12;
    c[2] = m00 * m20 + m01 * m21 + m02 * m22;
    c[3] = m10 * m10 + m11 * m11 + m12 * m12;
    c[4] = m10 * m20 + m11 * m21 + m12 * m22;
    c[5] = m20 * m20 + m21 * m21 + m22 * m22;
}

/* ---- ProjectiveJacobian.compute, src/math/projection.mojo:80-96 ---- */
template <typename T> static void jacobian(const V3<T>& t, T fx, T fy, T j[6]) {
    T tz = t.z;
    if (tz < (T)0.0001) tz = (T)0.0001;
    T inv_tz = T(1) / tz;
    T inv_tz2 = inv_tz * inv_tz;
    j[0] = fx * inv_tz; j[1] = T(0); j[2] = -fx * t.x * inv_tz2;
    j[3] = T(0); j[4] = fy * inv_tz; j[5] = -fy * t.y * inv_tz2;
}

/* ---- compute_ewa_covariance, src/math/projection.mojo:99-148 ---- */
template <typename T> static void ewa(const T s[6], const V3<T>& cam_pos, const M3<T>& W,
                                      T fx, T fy, T lowpass, T out[3]) {
    T J[6];
    jacobian(cam_pos, fx, fy, J);
    T t00 = J[0] * W.m00 + J[2] * W.m20;
    T t01 = J[0] * W.m01 + J[2] * W.m21;
    T t02 = J[0] * W.m02 + J[2] * W.m22;
    T t10 = J[4] * W.m10 + J[5] * W.m20;
    T t11 = J[4] * W.m11 + J[5] * W.m21;
    T t12 = J[4] * W.m12 + J[5] * W.m22;
    T s00 = s[0], s01 = s[1], s02 = s[2], s11 = s[3], s12 = s[4], s22 = s[5];
    T q00 = t00 * s00 + t01 * s01 + t02 * s02;
    T q01 = t00 * s01 + t01 * s11 + t02 * s12;
    T q02 = t00 * s02 + t01 * s12 + t02 * s22;
    T q10 = t10 * s00 + t11 * s01 + t12 * s02;
    T q11 = t10 * s01 + t11 * s11 + t12 * s12;
    T q12 = t10 * s02 + t11 * s12 + t12 * s22;
    out[0] = q00 * t00 + q01 * t01 + q02 * t02 + lowpass;
    out[1] = q00 * t10 + q01 * t11 + q02 * t12;
    out[2] = q10 * t10 + q11 * t11 + q12 * t12 + lowpass;
}

/* ---- Covariance2D.inverse, src/math/projection.mojo:30-42 ---- */
template <typename T> static void cov2_inverse(const T c[3], T out[3]) {
    T det = c[0] * c[2] - c[1] * c[1];
    if (det > (T)-0.0000001 && det < (T)0.0000001) { out[0] = out[1] = out[2] = T(0); return; }
    T inv_det = T(1) / det;
    out[0] = c[2] * inv_det;
    out[1] = -c[1] * inv_det;
    out[2] = c[0] * inv_det;
}

/* ---- solve_eigenvalues_2x2, src/math/cholesky.mojo:28-51 ---- */
template <typename T> static int64_t eigen_radius(const T c[3], T* lmax, T* lmin) {
    T a = c[0], b = c[1], cc = c[2];
    T mid = (a + cc) * (T)0.5;
    T diff = (a - cc) * (T)0.5;
    T disc = diff * diff + b * b;
    T root = std::sqrt(disc);
    T l_max = mid + root;
    T l_min = mid - root;
    if (l_min < T(0)) l_min = T(0);
    T r_float = (T)3.0 * std::sqrt(l_max);
    if (lmax) *lmax = l_max;
    if (lmin) *lmin = l_min;
    return mojo_int(std::ceil(r_float));
}

/* ---- SHBasis.evaluate, src/math/spherical_harmonics.mojo:17-26,68-111 ---- */
template <typename T> static void sh_basis(const V3<T>& dir, T y[16]) {
    const T C0 = (T)0.28209479177387814, C1 = (T)0.4886025119029199;
    const T C2_0 = (T)1.0925484305920792, C2_1 = (T)0.31539156525252005, C2_2 = (T)0.5462742152960396;
    const T C3_0 = (T)0.5900435899266435, C3_1 = (T)2.890611442640554, C3_2 = (T)0.4570457994644658;
    const T C3_3 = (T)0.3731763325901154, C3_4 = (T)1.445305721320277;
    V3<T> d = dir.normalized();
    T x = d.x, yv = d.y, z = d.z;
    T xx = x * x, yy = yv * yv, zz = z * z, xy = x * yv, yz = yv * z, xz = x * z;
    y[0] = C0;
    y[1] = -C1 * yv;
    y[2] = C1 * z;
    y[3] = -C1 * x;
    y[4] = C2_0 * xy;
    y[5] = -C2_0 * yz;
    y[6] = C2_1 * ((T)2.0 * zz - xx - yy);
    y[7] = -C2_0 * xz;
    y[8] = C2_2 * (xx - yy);
    y[9] = -C3_0 * yv * ((T)3.0 * xx - yy);
    y[10] = C3_1 * xy * z;
    y[11] = -C3_2 * yv * ((T)4.0 * zz - xx - yy);
    y[12] = C3_3 * z * ((T)2.0 * zz - (T)3.0 * xx - (T)3.0 * yy);
    y[13] = -C3_2 * x * ((T)4.0 * zz - xx - yy);
    y[14] = C3_4 * z * (xx - yy);
    y[15] = -C3_0 * x * (xx - (T)3.0 * yy);
}

/* ---- evaluate_sh_color, src/math/spherical_harmonics.mojo:133-172 ---- */
template <typename T> static void sh_color(const T* sh, const V3<T>& dir, int degree, T rgb[3],
                                           uint32_t* clamp_bits) {
    T y[16];
    sh_basis(dir, y);
    int max_coeffs = 16;
    if (degree == 0) max_coeffs = 1;
    else if (degree == 1) max_coeffs = 4;
    else if (degree == 2) max_coeffs = 9;
    T r = (T)0.5, g = (T)0.5, b = (T)0.5;
    for (int i = 0; i < max_coeffs; ++i) {
        T yv = y[i];
        r += sh[i * 3 + 0] * yv;
        g += sh[i * 3 + 1] * yv;
        b += sh[i * 3 + 2] * yv;
    }
    uint32_t cb = 0;
    if (r < T(0)) { r = T(0); cb |= 1; } else if (r > T(1)) { r = T(1); cb |= 2; }
    if (g < T(0)) { g = T(0); cb |= 4; } else if (g > T(1)) { g = T(1); cb |= 8; }
    if (b < T(0)) { b = T(0); cb |= 16; } else if (b > T(1)) { b = T(1); cb |= 32; }
    rgb[0] = r; rgb[1] = g; rgb[2] = b;
    if (clamp_bits) *clamp_bits = cb;
}

/* ---- float_to_ordered_uint32 / encode_tile_depth_key, radix_sort.mojo:8-27 ---- */
template <typename T> static uint64_t depth_bits(T z, int key_mode) {
    if (key_mode == 1) {
        float f = (float)z;
        uint32_t u;
        std::memcpy(&u, &f, 4);
        return (uint64_t)u;
    }
    int64_t scaled = mojo_int(z * (T)1000.0);
    if (scaled < 0) scaled = 0;
    else if (scaled > 0x7FFFFFFF) scaled = 0x7FFFFFFF;
    return (uint64_t)scaled;
}

/* ---- one Gaussian through pipeline.mojo:84-149 ---- */
template <typename T> struct Proj {
    bool visible;
    T cx, cy, z;
    T ic[3];
    T rgb[3];
    T op;
    int64_t radius;
    int64_t min_tx, min_ty, max_tx, max_ty;
    uint32_t sh_clamp;
};

template <typename T> static T act_opacity(T logit) {     /* gaussian.mojo:43-44 */
    return T(1) / (T(1) + Num<T>::exp(-logit));
}

template <typename T>
static Proj<T> project_one(int64_t i, const T* means, const T* scales, const T* quats,
                           const T* opac, const T* sh, const Cam<T>& cam, const M3<T>& view_rot,
                           const OracleOptions& o, int64_t tiles_x, int64_t tiles_y, int64_t ts) {
    Proj<T> p{};
    p.visible = false;
    p.radius = 0;
    /* get_gaussian + Gaussian3D.__init__ (normalises rotation), gaussian.mojo:109-114,36 */
    V3<T> pos{means[i * 3 + 0], means[i * 3 + 1], means[i * 3 + 2]};
    V3<T> scale{scales[i * 3 + 0], scales[i * 3 + 1], scales[i * 3 + 2]};
    T op = opac[i];
    if (o.params_are_logits) {
        scale = {Num<T>::exp(scale.x), Num<T>::exp(scale.y), Num<T>::exp(scale.z)};
        op = act_opacity(op);
    }
    Q<T> rot = Q<T>{quats[i * 4 + 0], quats[i * 4 + 1], quats[i * 4 + 2], quats[i * 4 + 3]}.normalized();
    /* culling.mojo:47-51 */
    if (!(op >= K<T>::min_alpha())) return p;
    V3<T> p_cam = cam.world_to_cam(pos);
    /* culling.mojo:41-45 */
    if (!(p_cam.z >= cam.near_plane && p_cam.z <= cam.far_plane)) return p;
    T sx, sy;
    cam.cam_to_screen(p_cam, sx, sy);
    T c3[6];
    cov3d(scale, rot, c3);
    T c2[3];
    ewa(c3, p_cam, view_rot, cam.fx, cam.fy, (T)o.lowpass, c2);
    int64_t radius = eigen_radius(c2, (T*)nullptr, (T*)nullptr);
    p.radius = radius;
    if (radius < 1) { p.radius = 0; return p; }
    /* is_screen_box_visible, culling.mojo:53-71 */
    T r_f = (T)radius;
    if (sx + r_f < T(0) || sx - r_f >= (T)cam.width || sy + r_f < T(0) || sy - r_f >= (T)cam.height) {
        p.radius = 0;
        return p;
    }
    /* get_gaussian_tile_overlap, tile.mojo:62-97 */
    int64_t min_px = mojo_int(sx - r_f), max_px = mojo_int(sx + r_f);
    int64_t min_py = mojo_int(sy - r_f), max_py = mojo_int(sy + r_f);
    if (max_px < 0 || min_px >= cam.width || max_py < 0 || min_py >= cam.height) {
        p.radius = 0;
        return p;
    }
    if (min_px < 0) min_px = 0;
    if (max_px >= cam.width) max_px = cam.width - 1;
    if (min_py < 0) min_py = 0;
    if (max_py >= cam.height) max_py = cam.height - 1;
    p.min_tx = min_px / ts; p.max_tx = max_px / ts;
    p.min_ty = min_py / ts; p.max_ty = max_py / ts;
    (void)tiles_x; (void)tiles_y;
    /* view direction and colour, pipeline.mojo:133-139 */
    V3<T> view_dir = pos.sub(cam.position).normalized();
    sh_color(sh + i * 48, view_dir, o.sh_degree, p.rgb, &p.sh_clamp);
    p.cx = sx; p.cy = sy; p.z = p_cam.z;
    cov2_inverse(c2, p.ic);
    p.op = op;
    p.visible = true;
    return p;
}

/* ---- radix_sort_64bit, radix_sort.mojo:39-87 (literal, single thread) ---- */
static void radix_sort_literal(uint64_t* keys, uint32_t* vals, int64_t n) {
    if (n <= 1) return;
    std::vector<uint64_t> kt(n);
    std::vector<uint32_t> vt(n);
    for (int pass = 0; pass < 8; ++pass) {
        int shift = pass * 8;
        int64_t counts[256] = {0};
        for (int64_t i = 0; i < n; ++i) counts[(keys[i] >> shift) & 0xFF]++;
        int64_t offsets[256];
        int64_t total = 0;
        for (int b = 0; b < 256; ++b) { offsets[b] = total; total += counts[b]; }
        for (int64_t i = 0; i < n; ++i) {
            uint64_t k = keys[i];
            uint32_t v = vals[i];
            int64_t d = offsets[(k >> shift) & 0xFF]++;
            kt[d] = k;
            vt[d] = v;
        }
        for (int64_t i = 0; i < n; ++i) { keys[i] = kt[i]; vals[i] = vt[i]; }
    }
}

/* Same stable LSD sort, 8 passes, with per-thread histograms over contiguous
 * chunks (chunks scattered in order keep the pass stable). */
static void radix_sort_parallel(uint64_t* keys, uint32_t* vals, int64_t n, int nt) {
    if (n <= 1) return;
    std::vector<uint64_t> kt(n);
    std::vector<uint32_t> vt(n);
    std::vector<int64_t> hist((size_t)nt * 256);
    uint64_t* src_k = keys; uint32_t* src_v = vals;
    uint64_t* dst_k = kt.data(); uint32_t* dst_v = vt.data();
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = pass * 8;
        std::fill(hist.begin(), hist.end(), 0);
        parallel_for(n, nt, [&](int64_t lo, int64_t hi, int t) {
            int64_t* h = &hist[(size_t)t * 256];
            for (int64_t i = lo; i < hi; ++i) h[(src_k[i] >> shift) & 0xFF]++;
        });
        int64_t total = 0;
        for (int b = 0; b < 256; ++b)
            for (int t = 0; t < nt; ++t) {
                int64_t c = hist[(size_t)t * 256 + b];
                hist[(size_t)t * 256 + b] = total;
                total += c;
            }
        parallel_for(n, nt, [&](int64_t lo, int64_t hi, int t) {
            int64_t* h = &hist[(size_t)t * 256];
            for (int64_t i = lo; i < hi; ++i) {
                uint64_t k = src_k[i];
                int64_t d = h[(k >> shift) & 0xFF]++;
                dst_k[d] = k;
                dst_v[d] = src_v[i];
            }
        });
        std::swap(src_k, dst_k);
        std::swap(src_v, dst_v);
    }
    /* 8 passes: the result is back in the caller's buffers */
}

/* ---- TileRangeIndex.build_from_sorted_keys, binning.mojo:51-73 ---- */
static void tile_ranges(const uint64_t* keys, int64_t n, int64_t total, int32_t* ranges) {
    for (int64_t t = 0; t < total; ++t) { ranges[2 * t] = -1; ranges[2 * t + 1] = -1; }
    if (n == 0) return;
    int64_t prev = -1;
    for (int64_t i = 0; i < n; ++i) {
        int64_t cur = (int64_t)((keys[i] >> 32) & 0xFFFFFFFFull);
        if (cur != prev) {
            if (prev >= 0 && prev < total) ranges[2 * prev + 1] = (int32_t)i;
            if (cur < total) { ranges[2 * cur] = (int32_t)i; ranges[2 * cur + 1] = (int32_t)n; }
            prev = cur;
        }
    }
    if (prev >= 0 && prev < total) ranges[2 * prev + 1] = (int32_t)n;
}

/* ---- compute_gaussian_pixel_alpha, compositor.mojo:62-89 ----
 * flags: 1 = beyond the 4.5 cutoff, 2 = clamped to 0.99, 4 = power clamped to 0 */
template <typename T> static T pixel_alpha(T px, T py, T cx, T cy, const T ic[3], T op, uint32_t* flags) {
    T dx = px - cx;
    T dy = py - cy;
    T power = (T)0.5 * (ic[0] * dx * dx + (T)2.0 * ic[1] * dx * dy + ic[2] * dy * dy);
    uint32_t f = 0;
    if (power < T(0)) { power = T(0); f |= 4; }
    else if (power > (T)4.5) { if (flags) *flags = 1; return T(0); }
    T g = Num<T>::exp(-power);
    T alpha = op * g;
    if (alpha > (T)0.99) { alpha = (T)0.99; f |= 2; }
    if (flags) *flags = f;
    return alpha;
}

struct Fnv {
    uint64_t h = 1469598103934665603ull;
    void add(uint64_t v) {
        for (int i = 0; i < 8; ++i) { h ^= (v >> (8 * i)) & 0xFF; h *= 1099511628211ull; }
    }
};

/* ---- the per-pixel compositing loop, pipeline.mojo:194-229 with
 * PixelAccumulator.blend/finalize, compositor.mojo:10-59 ---- */
template <typename T>
static void composite_tile(int64_t tx, int64_t ty, int64_t ts, int64_t W, int64_t H,
                           const int32_t* ranges, int64_t tiles_x, const uint32_t* vals,
                           const std::vector<Proj<T>>& rec, const OracleOptions& o,
                           T* rgb, T* depth, T* alpha_out, uint32_t* n_contrib, int32_t* last_idx,
                           Fnv* hash) {
    int64_t tile_id = ty * tiles_x + tx;
    int32_t rs = ranges[2 * tile_id], re = ranges[2 * tile_id + 1];
    int64_t px0 = tx * ts, px1 = std::min((tx + 1) * ts, W);
    int64_t py0 = ty * ts, py1 = std::min((ty + 1) * ts, H);
    bool empty = (rs == -1 || rs >= re);
    /* is_saturated threshold: TRANSMITTANCE_EPSILON (types.mojo:35) unless overridden */
    const T thr = (T)o.term_threshold;
    if (empty) {
        for (int64_t py = py0; py < py1; ++py)
            for (int64_t px = px0; px < px1; ++px) {
                int64_t p = py * W + px;
                if (o.white_background) { rgb[p * 3] = T(1); rgb[p * 3 + 1] = T(1); rgb[p * 3 + 2] = T(1); }
                if (alpha_out) alpha_out[p] = T(0);
                if (n_contrib) n_contrib[p] = 0;
                if (last_idx) last_idx[p] = -1;
            }
        return;
    }
    for (int64_t py = py0; py < py1; ++py) {
        T pyc = (T)py + (T)0.5;
        for (int64_t px = px0; px < px1; ++px) {
            T pxc = (T)px + (T)0.5;
            T cr = T(0), cg = T(0), cb = T(0), acc_alpha = T(0), Tr = T(1), d = T(0);
            uint32_t count = 0;
            int32_t last = -1;
            for (int32_t inst = rs; inst < re; ++inst) {
                const Proj<T>& g = rec[vals[inst]];
                last = inst;
                uint32_t fl = 0;
                T a = pixel_alpha(pxc, pyc, g.cx, g.cy, g.ic, g.op, &fl);
                /* blend, compositor.mojo:25-53 */
                if (a < K<T>::min_alpha()) {
                    if (hash && !(fl & 1)) { hash->add((uint64_t)inst << 8 | 0x10 | fl); }
                    continue;
                }
                T w = a * Tr;
                cr += g.rgb[0] * w;
                cg += g.rgb[1] * w;
                cb += g.rgb[2] * w;
                d += g.z * w;
                Tr *= (T(1) - a);
                acc_alpha = T(1) - Tr;
                count++;
                if (hash) hash->add((uint64_t)inst << 8 | 0x20 | fl);
                bool sat = (o.term_mode == 1) ? (acc_alpha >= thr) : (Tr <= thr);
                if (sat) break;
            }
            /* finalize, compositor.mojo:55-59 */
            if (o.white_background) { cr += Tr; cg += Tr; cb += Tr; }
            int64_t p = py * W + px;
            rgb[p * 3 + 0] = cr; rgb[p * 3 + 1] = cg; rgb[p * 3 + 2] = cb;
            if (o.compute_depth && depth) depth[p] = d;
            if (alpha_out) alpha_out[p] = acc_alpha;
            if (n_contrib) n_contrib[p] = count;
            if (last_idx) last_idx[p] = last;
            if (hash) hash->add(0xABCDEFull ^ (uint64_t)p);
        }
    }
}

template <typename T>
static int render_impl(const T* means, const T* scales, const T* quats, const T* opac, const T* sh,
                       int64_t n, const OracleCamera* ocam, const OracleOptions* o,
                       T* rgb, T* depth, T* alpha, uint32_t* n_contrib, int32_t* last_idx,
                       OracleOutputs* stages, uint64_t* decision_hash, int nt) {
    const int64_t W = ocam->width, H = ocam->height, ts = o->tile_size > 0 ? o->tile_size : 16;
    const int64_t P = W * H;
    /* RenderOutput: rgb and depth start at 0 (pipeline.mojo:29-35) */
    for (int64_t p = 0; p < P; ++p) {
        rgb[p * 3] = rgb[p * 3 + 1] = rgb[p * 3 + 2] = T(0);
        if (depth) depth[p] = T(0);
        if (alpha) alpha[p] = T(0);
        if (n_contrib) n_contrib[p] = 0;
        if (last_idx) last_idx[p] = -1;
    }
    const int64_t tiles_x = (W + ts - 1) / ts, tiles_y = (H + ts - 1) / ts, T_total = tiles_x * tiles_y;
    Fnv hash;
    int status = 0;
    if (stages) { stages->n_visible = 0; stages->n_instances = 0; }
    if (stages && stages->radii) for (int64_t i = 0; i < n; ++i) stages->radii[i] = 0;
    if (stages && stages->ranges) tile_ranges(nullptr, 0, T_total, stages->ranges);
    if (n == 0) { if (decision_hash) *decision_hash = hash.h; return 0; }   /* pipeline.mojo:64-65 */

    Cam<T> cam(*ocam);
    M3<T> view_rot = cam.view_rotation();

    /* 1. geometry and culling, pipeline.mojo:84-157 */
    std::vector<Proj<T>> proj(n);
    parallel_for(n, nt, [&](int64_t lo, int64_t hi, int) {
        for (int64_t i = lo; i < hi; ++i)
            proj[i] = project_one(i, means, scales, quats, opac, sh, cam, view_rot, *o, tiles_x, tiles_y, ts);
    });

    std::vector<Proj<T>> rec;
    rec.reserve(n);
    std::vector<uint64_t> keys;
    std::vector<uint32_t> vals;
    for (int64_t i = 0; i < n; ++i) {
        const Proj<T>& p = proj[i];
        if (stages && stages->radii) stages->radii[i] = p.visible ? (int32_t)std::min<int64_t>(p.radius, INT32_MAX) : 0;
        if (decision_hash) { hash.add((uint64_t)i); hash.add((uint64_t)p.visible); }
        if (!p.visible) continue;
        uint32_t vis = (uint32_t)rec.size();
        rec.push_back(p);
        if (decision_hash) {
            hash.add((uint64_t)p.radius); hash.add(p.sh_clamp);
            hash.add((uint64_t)p.min_tx); hash.add((uint64_t)p.max_tx);
            hash.add((uint64_t)p.min_ty); hash.add((uint64_t)p.max_ty);
        }
        uint64_t dk = depth_bits(p.z, o->key_mode);
        for (int64_t ty = p.min_ty; ty <= p.max_ty; ++ty)
            for (int64_t tx = p.min_tx; tx <= p.max_tx; ++tx) {
                uint64_t tile_id = (uint64_t)(ty * tiles_x + tx);
                keys.push_back((tile_id << 32) | dk);
                vals.push_back(vis);
            }
    }
    const int64_t V = (int64_t)rec.size(), Kn = (int64_t)keys.size();
    if (stages) {
        stages->n_visible = V;
        stages->n_instances = Kn;
        if (stages->records) {
            if (stages->records_cap >= V) {
                for (int64_t v = 0; v < V; ++v) {
                    const Proj<T>& p = rec[v];
                    OracleRecord& r = stages->records[v];
                    r.cx = (float)p.cx; r.cy = (float)p.cy; r.depth = (float)p.z;
                    r.ic00 = (float)p.ic[0]; r.ic01 = (float)p.ic[1]; r.ic11 = (float)p.ic[2];
                    r.r = (float)p.rgb[0]; r.g = (float)p.rgb[1]; r.b = (float)p.rgb[2];
                    r.opacity = (float)p.op;
                }
            } else status = -1;
        }
        if (stages->keys_unsorted && stages->vals_unsorted) {
            if (stages->keys_cap >= Kn) {
                std::memcpy(stages->keys_unsorted, keys.data(), Kn * sizeof(uint64_t));
                std::memcpy(stages->vals_unsorted, vals.data(), Kn * sizeof(uint32_t));
            } else status = -1;
        }
    }
    if (Kn == 0) { if (decision_hash) *decision_hash = hash.h; return status; }   /* pipeline.mojo:162-163 */

    /* 2. sort, pipeline.mojo:166 */
    if (nt > 1) radix_sort_parallel(keys.data(), vals.data(), Kn, nt);
    else radix_sort_literal(keys.data(), vals.data(), Kn);
    if (decision_hash) for (int64_t i = 0; i < Kn; ++i) hash.add(vals[i]);

    /* 3. ranges, pipeline.mojo:169 */
    std::vector<int32_t> ranges((size_t)T_total * 2);
    tile_ranges(keys.data(), Kn, T_total, ranges.data());
    if (stages) {
        if (stages->keys_sorted && stages->vals_sorted) {
            if (stages->keys_cap >= Kn) {
                std::memcpy(stages->keys_sorted, keys.data(), Kn * sizeof(uint64_t));
                std::memcpy(stages->vals_sorted, vals.data(), Kn * sizeof(uint32_t));
            } else status = -1;
        }
        if (stages->ranges) std::memcpy(stages->ranges, ranges.data(), ranges.size() * sizeof(int32_t));
    }

    /* 4. compositing, pipeline.mojo:172-229 */
    if (decision_hash) {
        for (int64_t ty = 0; ty < tiles_y; ++ty)
            for (int64_t tx = 0; tx < tiles_x; ++tx)
                composite_tile(tx, ty, ts, W, H, ranges.data(), tiles_x, vals.data(), rec, *o,
                               rgb, depth, alpha, n_contrib, last_idx, &hash);
        *decision_hash = hash.h;
    } else {
        parallel_dynamic(T_total, nt, 4, [&](int64_t t) {
            composite_tile(t % tiles_x, t / tiles_x, ts, W, H, ranges.data(), tiles_x, vals.data(), rec, *o,
                           rgb, depth, alpha, n_contrib, last_idx, (Fnv*)nullptr);
        });
    }
    return status;
}

}  // namespace

extern "C" {

int oracle_render_f32(const float* means, const float* scales, const float* quats,
                      const float* opacities, const float* sh, int64_t n,
                      const OracleCamera* cam, const OracleOptions* opt,
                      OracleOutputs* out, int nthreads) {
    return render_impl<float>(means, scales, quats, opacities, sh, n, cam, opt,
                              out->rgb, out->depth, out->alpha, out->n_contrib, out->last_idx,
                              out, nullptr, nthreads);
}

int oracle_render_f64(const double* means, const double* scales, const double* quats,
                      const double* opacities, const double* sh, int64_t n,
                      const OracleCamera* cam, const OracleOptions* opt,
                      double* rgb, double* depth, double* alpha, uint64_t* decision_hash) {
    return render_impl<double>(means, scales, quats, opacities, sh, n, cam, opt,
                               rgb, depth, alpha, nullptr, nullptr, nullptr, decision_hash, 1);
}

void oracle_radix_sort64(uint64_t* keys, uint32_t* vals, int64_t n, int nthreads) {
    if (nthreads > 1) radix_sort_parallel(keys, vals, n, nthreads);
    else radix_sort_literal(keys, vals, n);
}

void oracle_tile_ranges(const uint64_t* keys, int64_t n, int64_t total_tiles, int32_t* ranges) {
    tile_ranges(keys, n, total_tiles, ranges);
}

uint64_t oracle_encode_key(uint32_t tile_id, float depth, int key_mode) {
    return ((uint64_t)tile_id << 32) | depth_bits<float>(depth, key_mode);
}

float oracle_l1_loss(const float* pred, const float* target, int64_t n, float* grad) {
    if (n == 0) return 0.0f;                        /* loss.mojo:20-21 */
    float sum = 0.0f;
    float inv_n = 1.0f / (float)n;
    for (int64_t i = 0; i < n; ++i) {
        float diff = pred[i] - target[i];
        if (diff >= 0.0f) { sum += diff; if (grad) grad[i] = inv_n; }
        else { sum -= diff; if (grad) grad[i] = -inv_n; }
    }
    return sum * inv_n;
}

void oracle_ewa_cov2d(const float c3[6], const float t[3], const float vr[9], float fx, float fy,
                      float lowpass, float out[3]) {
    M3<float> W{vr[0], vr[1], vr[2], vr[3], vr[4], vr[5], vr[6], vr[7], vr[8]};
    ewa<float>(c3, V3<float>{t[0], t[1], t[2]}, W, fx, fy, lowpass, out);
}

void oracle_jacobian(const float t[3], float fx, float fy, float out[6]) {
    jacobian<float>(V3<float>{t[0], t[1], t[2]}, fx, fy, out);
}

void oracle_cov3d(const float s[3], const float q[4], float out[6]) {
    cov3d<float>(V3<float>{s[0], s[1], s[2]}, Q<float>{q[0], q[1], q[2], q[3]}, out);
}

void oracle_eigen2x2(const float c[3], float out[2], int64_t* radius) {
    *radius = eigen_radius<float>(c, &out[0], &out[1]);
}

void oracle_cov2d_inverse(const float c[3], float out[3]) { cov2_inverse<float>(c, out); }

void oracle_sh_basis(const float d[3], float out[16]) { sh_basis<float>(V3<float>{d[0], d[1], d[2]}, out); }

void oracle_sh_color(const float* sh48, const float d[3], int degree, float out[3]) {
    sh_color<float>(sh48, V3<float>{d[0], d[1], d[2]}, degree, out, nullptr);
}

int oracle_depth_visible(float z, float near_plane, float far_plane) {
    return z >= near_plane && z <= far_plane;
}

int oracle_screen_box_visible(float cx, float cy, int64_t radius, int32_t w, int32_t h) {
    float r_f = (float)radius;
    if (cx + r_f < 0.0f) return 0;
    if (cx - r_f >= (float)w) return 0;
    if (cy + r_f < 0.0f) return 0;
    if (cy - r_f >= (float)h) return 0;
    return 1;
}

void oracle_world_to_screen(const OracleCamera* c, const float p[3], float out_cam[3], float out_screen[2]) {
    Cam<float> cam(*c);
    V3<float> pc = cam.world_to_cam(V3<float>{p[0], p[1], p[2]});
    out_cam[0] = pc.x; out_cam[1] = pc.y; out_cam[2] = pc.z;
    cam.cam_to_screen(pc, out_screen[0], out_screen[1]);
}

int oracle_blend_sequence(const float* colors, const float* alphas, const float* depths, int n,
                          int term_mode, float out_color[3], float* out_T, float* out_depth,
                          float* out_alpha) {
    float cr = 0, cg = 0, cb = 0, a_acc = 0, Tr = 1, d = 0;
    int term = 0;
    for (int i = 0; i < n; ++i) {
        float a = alphas[i];
        term = 0;
        if (a < K<float>::min_alpha()) continue;
        float w = a * Tr;
        cr += colors[i * 3] * w; cg += colors[i * 3 + 1] * w; cb += colors[i * 3 + 2] * w;
        d += depths[i] * w;
        Tr *= (1.0f - a);
        a_acc = 1.0f - Tr;
        term = (term_mode == 1) ? (a_acc >= 0.99f) : (Tr <= K<float>::t_eps());
    }
    out_color[0] = cr; out_color[1] = cg; out_color[2] = cb;
    *out_T = Tr; *out_depth = d; *out_alpha = a_acc;
    return term;
}

float oracle_pixel_alpha(float px, float py, float cx, float cy, const float ic[3], float op) {
    return pixel_alpha<float>(px, py, cx, cy, ic, op, nullptr);
}

}  // extern "C"
