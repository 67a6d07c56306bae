// Daylight on the host: the Preetham sky map and the sun's spectral radiance that PRender builds
// for a "sun_sky" light (src/scene/scene_loader.cpp:977-996), restated so that a caller without
// PRender's scene classes can light a scene the same way, plus the fit of RGB texels to
// sigmoid-polynomial spectra that the module's environment maps take.
//
//   prhost_preetham_sky   -- pr::MakePreethamSky (src/lights/sky.cpp:146-205): Perez luminance and
//                            chromaticity distributions (A. J. Preetham, P. Shirley, B. Smits, "A
//                            Practical Analytic Model for Daylight", SIGGRAPH 1999) at turbidity T,
//                            zenith values from the paper's fits, converted to linear sRGB, a
//                            Lambertian ground below the horizon lit by sky and sun.
//   prhost_sun_radiance   -- pr::MakeSunRadiance (src/lights/sky.cpp:207-233): a 5778 K blackbody
//                            scaled to the solar disk's luminance, attenuated by Rayleigh and
//                            Angstrom aerosol optical depth over the Kasten-Young (1989) air mass.
//   prhost_rgb_to_sigmoid -- per texel, the sigmoid polynomial S(c0 l^2 + c1 l + c2) (l in nm) and
//                            scale 2 max(r, g, b) of an unbounded RGB (the representation of
//                            RGBUnboundedSpectrum, src/core/rgb2spec.cpp:327-335), fitted by
//                            Gauss-Newton in CIELAB under a caller-given illuminant (W. Jakob,
//                            J. Hanika, "A Low-Dimensional Function Space for Efficient Spectral
//                            Upsampling", 2019). The reference instead interpolates a precomputed
//                            64^3 table of the same fits under CIE D65.
//
// Arithmetic follows the reference in FP32 with the same operation order (the 1 nm spectrum
// integrals in FP64), so the sky and sun agree with it to rounding.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "prhost_api.h"

namespace {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;

float clampf(float v, float lo, float hi) { return std::min(std::max(v, lo), hi); }
float radians(float deg) { return (kPi / 180.f) * deg; }
float degrees(float rad) { return (180.f / kPi) * rad; }
float safe_acos(float x) { return std::acos(clampf(x, -1.f, 1.f)); }
float safe_sqrt(float x) { return std::sqrt(std::max(0.f, x)); }
float smooth_step(float x, float a, float b) {
    if (a == b) return x < a ? 0.f : 1.f;
    float t = clampf((x - a) / (b - a), 0.f, 1.f);
    return t * t * (3 - 2 * t);
}

// CIE 1931 observer, the multi-lobe fit of Wyman, Sloan and Shirley (JCGT 2013).
float lobe(float x, float mu, float s1, float s2) {
    float t = (x - mu) / (x < mu ? s1 : s2);
    return std::exp(-0.5f * t * t);
}
float cie_x(float l) {
    return 1.056f * lobe(l, 599.8f, 37.9f, 31.0f) + 0.362f * lobe(l, 442.0f, 16.0f, 26.7f) -
           0.065f * lobe(l, 501.1f, 20.4f, 26.2f);
}
float cie_y(float l) { return 0.821f * lobe(l, 568.8f, 46.9f, 40.5f) + 0.286f * lobe(l, 530.9f, 16.3f, 31.1f); }
float cie_z(float l) { return 1.217f * lobe(l, 437.0f, 11.8f, 36.0f) + 0.681f * lobe(l, 459.0f, 26.0f, 13.8f); }

float cie_y_integral() {
    static const float v = [] {
        double s = 0;
        for (int l = 360; l <= 830; ++l) s += cie_y(float(l));
        return float(s);
    }();
    return v;
}

// Luminance of a spectrum: the 1 nm sum of CIE y times the spectrum over 360..830 nm.
template <typename F> float spectrum_y(F &&s) {
    double Y = 0;
    for (int l = 360; l <= 830; ++l) Y += cie_y(float(l)) * s(float(l));
    return float(Y) * (1.f / cie_y_integral());
}

float planck(float lambdaNm, float T) {
    if (T <= 0) return 0;
    const double c = 299792458., h = 6.62606957e-34, kb = 1.3806488e-23;
    double l = lambdaNm * 1e-9;
    return float((2 * h * c * c) / (std::pow(l, 5) * (std::exp((h * c) / (l * kb * T)) - 1)));
}

// Planck's law normalised to a peak of 1 (Wien's displacement law for the peak).
struct Blackbody {
    float T, norm;
    explicit Blackbody(float t) : T(t) { norm = 1 / planck(2.8977721e-3f / T * 1e9f, T); }
    float operator()(float l) const { return planck(l, T) * norm; }
};

// Piecewise-linear spectrum over ascending samples, constant beyond the ends.
struct Piecewise {
    std::vector<float> l, v;
    float operator()(float x) const {
        if (l.empty()) return 0;
        if (x <= l.front()) return v.front();
        if (x >= l.back()) return v.back();
        int lo = 0, n = int(l.size()) - 2;  // largest i <= n with l[i] <= x
        int hi = n;
        while (lo < hi) {
            int mid = (lo + hi + 1) / 2;
            if (l[mid] <= x) lo = mid;
            else hi = mid - 1;
        }
        float t = (x - l[lo]) / (l[lo + 1] - l[lo]);
        return (1 - t) * v[lo] + t * v[lo + 1];
    }
};

Piecewise sun_radiance(const float *sunDir, float T, float angularRadiusDeg) {
    float len = std::sqrt(sunDir[0] * sunDir[0] + sunDir[1] * sunDir[1] + sunDir[2] * sunDir[2]);
    float dy = sunDir[1] / len;
    float elevDeg = degrees(std::asin(clampf(dy, -1.f, 1.f)));
    float zenithDeg = 90 - elevDeg;
    float m = zenithDeg < 95 ? 1 / (std::cos(radians(std::min(zenithDeg, 90.f))) +
                                    0.50572f * std::pow(96.07995f - zenithDeg, -1.6364f))
                             : 1e3f;
    float beta = std::max(0.f, 0.04608f * T - 0.04586f);
    Blackbody bb(5778);
    float yBB = spectrum_y(bb);
    float r = std::max(angularRadiusDeg, 0.01f);
    float sizeScale = (0.2665f / r) * (0.2665f / r);
    Piecewise s;
    for (int lambda = 360; lambda <= 830; lambda += 5) {
        float um = lambda * 1e-3f;
        float tauR = 0.008735f * std::pow(um, -4.08f);
        float tauA = beta * std::pow(um, -1.3f);
        float trans = elevDeg < -1 ? 0.f : std::exp(-m * (tauR + tauA));
        s.l.push_back(float(lambda));
        s.v.push_back(2.0e6f * sizeScale * bb(float(lambda)) / yBB * trans);
    }
    return s;
}

struct Perez {
    float A, B, C, D, E;
    float F(float cosTheta, float gamma, float cosGamma) const {
        cosTheta = std::max(cosTheta, 0.01f);
        return (1 + A * std::exp(B / cosTheta)) * (1 + C * std::exp(D * gamma) + E * cosGamma * cosGamma);
    }
};

void equirect_dir(float u, float v, float *d) {
    float theta = v * kPi, phi = u * 2 * kPi;
    float s = std::sin(theta);
    d[0] = s * std::cos(phi);
    d[1] = std::cos(theta);
    d[2] = s * std::sin(phi);
}

// CIE XYZ -> linear sRGB (D65 white), the standard matrix.
constexpr float kXYZToSRGB[3][3] = {{3.2404542f, -1.5371385f, -0.4985314f},
                                    {-0.9692660f, 1.8760108f, 0.0415560f},
                                    {0.0556434f, -0.2040259f, 1.0572252f}};

// ---- RGB -> sigmoid polynomial ----

struct FitTables {
    std::vector<double> w[3];  // illuminant x CIE xyz at the quadrature wavelengths, Y of white = 1
};

double lab_f(double t) {
    const double d = 6.0 / 29.0;
    return t > d * d * d ? std::cbrt(t) : t / (3 * d * d) + 4.0 / 29.0;
}

void to_lab(const double *xyz, const double *white, double *lab) {
    double fx = lab_f(xyz[0] / white[0]), fy = lab_f(xyz[1] / white[1]), fz = lab_f(xyz[2] / white[2]);
    lab[0] = 116 * fy - 16;
    lab[1] = 500 * (fx - fy);
    lab[2] = 200 * (fy - fz);
}

double sigmoid(double x) { return 0.5 + x / (2.0 * std::sqrt(1.0 + x * x)); }

// XYZ of the reflectance S(c0 t^2 + c1 t + c2), t = (l - 360) / 470, under the fit illuminant.
void fit_xyz(const FitTables &T, const double *c, double *xyz) {
    xyz[0] = xyz[1] = xyz[2] = 0;
    const int n = int(T.w[0].size());
    for (int i = 0; i < n; ++i) {
        double t = double(i) / double(n - 1);
        double s = sigmoid((c[0] * t + c[1]) * t + c[2]);
        xyz[0] += T.w[0][i] * s;
        xyz[1] += T.w[1][i] * s;
        xyz[2] += T.w[2][i] * s;
    }
}

bool solve3(double A[3][3], double *b) {
    for (int c = 0; c < 3; ++c) {
        int p = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[p][c])) p = r;
        if (std::fabs(A[p][c]) < 1e-15) return false;
        for (int k = 0; k < 3; ++k) std::swap(A[c][k], A[p][k]);
        std::swap(b[c], b[p]);
        for (int r = 0; r < 3; ++r) {
            if (r == c) continue;
            double f = A[r][c] / A[c][c];
            for (int k = 0; k < 3; ++k) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int c = 0; c < 3; ++c) b[c] /= A[c][c];
    return true;
}

// Gauss-Newton on the CIELAB residual of a reflectance rgb in [0, 1]^3 (sRGB primaries), starting
// from c (zero: a flat 1/2). Returns c in normalised wavelength t.
void fit_one(const FitTables &T, const double rgb[3], double *c) {
    const double M[3][3] = {{0.4124564, 0.3575761, 0.1804375}, {0.2126729, 0.7151522, 0.0721750},
                            {0.0193339, 0.1191920, 0.9503041}};
    // Target: the colour's XYZ with the sRGB (D65) white point, in CIELAB relative to that white;
    // the reflectance's XYZ under the fit illuminant (unit luminance) is compared in the same
    // space, so an illuminant whose white differs from D65 is corrected for, not inherited.
    const double white[3] = {M[0][0] + M[0][1] + M[0][2], M[1][0] + M[1][1] + M[1][2], M[2][0] + M[2][1] + M[2][2]};
    double xyz[3], target[3];
    for (int i = 0; i < 3; ++i) xyz[i] = M[i][0] * rgb[0] + M[i][1] * rgb[1] + M[i][2] * rgb[2];
    to_lab(xyz, white, target);
    for (int it = 0; it < 40; ++it) {
        double cur[3], lab[3], r[3];
        fit_xyz(T, c, cur);
        to_lab(cur, white, lab);
        for (int i = 0; i < 3; ++i) r[i] = target[i] - lab[i];
        if (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < 1e-10) break;
        double J[3][3];
        for (int k = 0; k < 3; ++k) {
            double cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
            cp[k] += 1e-5;
            cm[k] -= 1e-5;
            double xp[3], xm[3], lp[3], lm[3];
            fit_xyz(T, cp, xp);
            fit_xyz(T, cm, xm);
            to_lab(xp, white, lp);
            to_lab(xm, white, lm);
            for (int i = 0; i < 3; ++i) J[i][k] = -(lp[i] - lm[i]) / 2e-5;  // d residual / d c
        }
        double step[3] = {r[0], r[1], r[2]};
        if (!solve3(J, step)) break;
        for (int k = 0; k < 3; ++k) c[k] -= step[k];
        double mx = std::max(std::fabs(c[0]), std::max(std::fabs(c[1]), std::fabs(c[2])));
        if (mx > 200) {
            for (int k = 0; k < 3; ++k) c[k] *= 200 / mx;
        }
    }
}

} // namespace

PRHOST_API int prhost_sun_radiance(const float *sunDir, float turbidity, float angularRadiusDeg, int64_t n,
                                   const float *lambdaNm, float *out) {
    if (!sunDir || n < 0 || (n > 0 && (!lambdaNm || !out))) return 1;
    Piecewise s = sun_radiance(sunDir, turbidity, angularRadiusDeg);
    for (int64_t i = 0; i < n; ++i) out[i] = s(lambdaNm[i]);
    return 0;
}

PRHOST_API int prhost_preetham_sky(const float *sunDirIn, float T, float groundAlbedo, int32_t width, int32_t height,
                                   float *rgb) {
    if (!sunDirIn || !rgb || width <= 0 || height <= 0) return 1;
    float len = std::sqrt(sunDirIn[0] * sunDirIn[0] + sunDirIn[1] * sunDirIn[1] + sunDirIn[2] * sunDirIn[2]);
    if (!(len > 0)) return 1;
    const float sun[3] = {sunDirIn[0] / len, sunDirIn[1] / len, sunDirIn[2] / len};
    T = clampf(T, 1.7f, 10.f);
    float thetaS = safe_acos(std::max(sun[1], 0.f));
    // Perez coefficients of luminance Y and chromaticities x, y as linear functions of T.
    Perez pY{0.1787f * T - 1.4630f, -0.3554f * T + 0.4275f, -0.0227f * T + 5.3251f, 0.1206f * T - 2.5771f,
             -0.0670f * T + 0.3703f};
    Perez px{-0.0193f * T - 0.2592f, -0.0665f * T + 0.0008f, -0.0004f * T + 0.2125f, -0.0641f * T - 0.8989f,
             -0.0033f * T + 0.0452f};
    Perez py{-0.0167f * T - 0.2608f, -0.0950f * T + 0.0092f, -0.0079f * T + 0.2102f, -0.0441f * T - 1.6537f,
             -0.0109f * T + 0.0529f};
    float chi = (4.f / 9.f - T / 120.f) * (kPi - 2 * thetaS);
    float Yz = std::max(0.f, (4.0453f * T - 4.9710f) * std::tan(chi) - 0.2155f * T + 2.4192f);
    float t2 = thetaS * thetaS, t3 = t2 * thetaS;
    float xz = T * T * (0.00166f * t3 - 0.00375f * t2 + 0.00209f * thetaS) +
               T * (-0.02903f * t3 + 0.06377f * t2 - 0.03202f * thetaS + 0.00394f) +
               (0.11693f * t3 - 0.21196f * t2 + 0.06052f * thetaS + 0.25886f);
    float yz = T * T * (0.00275f * t3 - 0.00610f * t2 + 0.00317f * thetaS) +
               T * (-0.04214f * t3 + 0.08970f * t2 - 0.04153f * thetaS + 0.00516f) +
               (0.15346f * t3 - 0.26756f * t2 + 0.06670f * thetaS + 0.26688f);
    float cosS = std::cos(thetaS);
    float denY = pY.F(1, thetaS, cosS), denx = px.F(1, thetaS, cosS), deny = py.F(1, thetaS, cosS);
    float night = smooth_step(sun[1], -0.1f, 0.02f);
    float up[3] = {sun[0], std::max(sun[1], 0.f), sun[2]};
    float ul = std::sqrt(up[0] * up[0] + up[1] * up[1] + up[2] * up[2]);
    for (float &v : up) v /= ul;
    double skyE = 0;
    for (int j = 0; j < height; ++j)
        for (int i = 0; i < width; ++i) {
            float w[3];
            equirect_dir((i + 0.5f) / width, (j + 0.5f) / height, w);
            float *c = rgb + 3 * (size_t(j) * width + i);
            c[0] = c[1] = c[2] = 0.f;
            if (w[1] > 0) {
                float cosG = clampf(w[0] * up[0] + w[1] * up[1] + w[2] * up[2], -1.f, 1.f);
                float gamma = std::acos(cosG);
                float Y = Yz * pY.F(w[1], gamma, cosG) / denY * night;
                float x = xz * px.F(w[1], gamma, cosG) / denx;
                float y = yz * py.F(w[1], gamma, cosG) / deny;
                if (y > 0 && Y > 0) {
                    float X = x / y * Y, Z = (1 - x - y) / y * Y;
                    for (int k = 0; k < 3; ++k)
                        c[k] = std::max(0.f, kXYZToSRGB[k][0] * X + kXYZToSRGB[k][1] * Y + kXYZToSRGB[k][2] * Z);
                    float dOmega = (2 * kPi / width) * (kPi / height) * safe_sqrt(1 - w[1] * w[1]);
                    skyE += Y * w[1] * dOmega;
                }
            }
        }
    float sunE = 0;
    if (sun[1] > 0) {
        const float r = radians(0.2665f);
        Piecewise s = sun_radiance(sun, T, 0.2665f);
        sunE = spectrum_y(s) * kPi * r * r * sun[1];
    }
    float groundY = groundAlbedo * kInvPi * (float(skyE) + sunE);
    for (int j = 0; j < height; ++j)
        for (int i = 0; i < width; ++i) {
            float w[3];
            equirect_dir((i + 0.5f) / width, (j + 0.5f) / height, w);
            if (w[1] <= 0) {
                float *c = rgb + 3 * (size_t(j) * width + i);
                c[0] = c[1] = c[2] = groundY;
            }
        }
    return 0;
}

PRHOST_API int prhost_rgb_to_sigmoid(int64_t n, const float *rgb, const float *illuminant95, int32_t threads,
                                     float *out4) {
    if (n < 0 || (n > 0 && (!rgb || !out4 || !illuminant95))) return 1;
    FitTables T;
    for (int i = 0; i < 95; ++i) {
        const float l = 360.f + 5.f * float(i);
        const double e = illuminant95[i];
        T.w[0].push_back(e * cie_x(l));
        T.w[1].push_back(e * cie_y(l));
        T.w[2].push_back(e * cie_z(l));
    }
    double ysum = 0;
    for (double v : T.w[1]) ysum += v;
    if (!(ysum > 0)) return 1;
    for (int k = 0; k < 3; ++k)
        for (double &v : T.w[k]) v /= ysum;
    int nt = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    nt = int(std::min<int64_t>(nt, std::max<int64_t>(1, n / 256)));
    auto work = [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            double c[3] = {0, 0, 0};  // every texel from the same start: results independent of threads
            const float *p = rgb + 3 * i;
            float m = std::max(0.f, std::max(p[0], std::max(p[1], p[2])));
            float *o = out4 + 4 * i;
            if (m == 0.f) {
                o[0] = o[1] = o[2] = o[3] = 0.f;
                continue;
            }
            float scale = 2 * m, inv = 1 / scale;
            double q[3] = {clampf(p[0] * inv, 0.f, 1.f), clampf(p[1] * inv, 0.f, 1.f), clampf(p[2] * inv, 0.f, 1.f)};
            fit_one(T, q, c);
            // S(c0 t^2 + c1 t + c2), t = (l - 360) / 470, as a polynomial in l.
            const double a = 1.0 / 470.0, b0 = -360.0 / 470.0;
            o[0] = float(c[0] * a * a);
            o[1] = float(2 * c[0] * a * b0 + c[1] * a);
            o[2] = float(c[0] * b0 * b0 + c[1] * b0 + c[2]);
            o[3] = scale;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) pool.emplace_back(work, n * t / nt, n * (t + 1) / nt);
    for (auto &th : pool) th.join();
    return 0;
}
