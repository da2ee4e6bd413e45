// synth.cpp — seeded synthetic luma sequences for the inter-analysis stage.
//
// The reference measures its encoder on FFmpeg lavfi clips (testsrc2, mandelbrot, a "noisy 720p
// clip"), none of which exist here; these sequences stand in for them with the shapes the stage's
// benchmark configurations name:
//   - background: 4-octave value noise (base period 64 px, amplitude halving per octave) mapped to
//     luma 16..235, sampled at (x + Px(t), y + Py(t)) where P(t) is the running sum of per-frame
//     quarter-sample pans drawn uniformly from [-pan_q, pan_q] / 4 px;
//   - nobj rectangles (sides 64..256 px, own noise texture) moving linearly at per-object velocities
//     uniform in [-vmax, vmax] px/frame rounded to quarter samples, wrapping around the picture;
//   - i.i.d. Gaussian sensor noise of standard deviation sigma, then rounding half away from zero
//     and clamping to 0..255.
// Only luma is produced: chroma is not read by the inter-analysis stage.
//
// Determinism: lattice values come from splitmix64 of (seed, octave, i, j); pans and objects from
// std::mt19937_64 streams (seed + 1, seed + 3); the sensor noise of frame t from a mt19937_64 seeded
// with (seed + 2) ^ (t * golden ratio), so any frame can be generated on its own.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline double lattice(uint64_t seed, int o, int64_t i, int64_t j) {
    uint64_t key = (seed << 40) ^ (uint64_t(o) << 32) ^ (uint64_t(uint16_t(j)) << 16) ^ uint64_t(uint16_t(i));
    return double(splitmix64(key) >> 32) * (1.0 / 4294967296.0);
}

inline double smooth(double f) { return f * f * (3.0 - 2.0 * f); }

// 4-octave value noise in [0, 1] at real coordinates.
double value_noise(uint64_t seed, double x, double y) {
    double sum = 0.0, norm = 0.0;
    for (int o = 0; o < 4; o++) {
        double p = double(64 >> o), amp = 1.0 / double(1 << o);
        double u = x / p, v = y / p;
        double fi = std::floor(u), fj = std::floor(v);
        int64_t i = int64_t(fi), j = int64_t(fj);
        double su = smooth(u - fi), sv = smooth(v - fj);
        double a = lattice(seed, o, i, j), b = lattice(seed, o, i + 1, j);
        double c = lattice(seed, o, i, j + 1), d = lattice(seed, o, i + 1, j + 1);
        double top = a + (b - a) * su, bot = c + (d - c) * su;
        sum += amp * (top + (bot - top) * sv);
        norm += amp;
    }
    return sum / norm;
}

inline double uniform01(std::mt19937_64& g) { return double(g() >> 11) * (1.0 / 9007199254740992.0); }

struct Obj {
    int w, h;
    double x0, y0, vx, vy;
    uint64_t seed;
};

struct Synth {
    int width, height;
    uint64_t seed;
    double sigma;
    std::vector<double> px, py;  // cumulative pan per frame, px
    std::vector<Obj> objs;
};

}  // namespace

extern "C" {

// Creates a generator for `frames` frames of width x height luma.
void* ironav_synth_create(int width, int height, int frames, uint64_t seed, int pan_q, int nobj, double vmax, double sigma) {
    if (width <= 0 || height <= 0 || frames <= 0 || pan_q < 0 || nobj < 0) return nullptr;
    Synth* s = new Synth();
    s->width = width;
    s->height = height;
    s->seed = seed;
    s->sigma = sigma;
    std::mt19937_64 pan(seed + 1);
    double cx = 0.0, cy = 0.0;
    for (int t = 0; t < frames; t++) {
        if (t > 0) {
            int dx = int(pan() % uint64_t(2 * pan_q + 1)) - pan_q;
            int dy = int(pan() % uint64_t(2 * pan_q + 1)) - pan_q;
            cx += dx * 0.25;
            cy += dy * 0.25;
        }
        s->px.push_back(cx);
        s->py.push_back(cy);
    }
    std::mt19937_64 og(seed + 3);
    for (int k = 0; k < nobj; k++) {
        Obj o;
        o.w = 64 + int(og() % 193);
        o.h = 64 + int(og() % 193);
        o.x0 = uniform01(og) * width;
        o.y0 = uniform01(og) * height;
        o.vx = std::round((uniform01(og) * 2.0 - 1.0) * vmax * 4.0) / 4.0;
        o.vy = std::round((uniform01(og) * 2.0 - 1.0) * vmax * 4.0) / 4.0;
        o.seed = splitmix64(seed ^ (0xA24BAED4963EE407ull * uint64_t(k + 1)));
        s->objs.push_back(o);
    }
    return s;
}

void ironav_synth_destroy(void* h) { delete static_cast<Synth*>(h); }

// Writes frame t (width x height, rows `stride` bytes apart).
int ironav_synth_frame(void* h, int t, uint8_t* out, int stride) {
    Synth* s = static_cast<Synth*>(h);
    if (!s || !out || t < 0 || t >= int(s->px.size()) || stride < s->width) return 3;
    const int W = s->width, H = s->height;
    std::vector<double> img(size_t(W) * H);
    const double ox = s->px[t], oy = s->py[t];
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) img[size_t(y) * W + x] = value_noise(s->seed, x + ox, y + oy);
    for (const Obj& o : s->objs) {
        // position wraps around the picture so objects keep crossing it
        double spanx = W + o.w, spany = H + o.h;
        double xt = std::fmod(o.x0 + o.vx * t + o.w, spanx);
        if (xt < 0) xt += spanx;
        double yt = std::fmod(o.y0 + o.vy * t + o.h, spany);
        if (yt < 0) yt += spany;
        xt -= o.w;
        yt -= o.h;
        int xa = std::max(0, int(std::ceil(xt))), xb = std::min(W, int(std::ceil(xt + o.w)));
        int ya = std::max(0, int(std::ceil(yt))), yb = std::min(H, int(std::ceil(yt + o.h)));
#pragma omp parallel for schedule(static)
        for (int y = ya; y < yb; y++)
            for (int x = xa; x < xb; x++) img[size_t(y) * W + x] = value_noise(o.seed, x - xt, y - yt);
    }
    std::mt19937_64 ng((s->seed + 2) ^ (uint64_t(t) * 0x9E3779B97F4A7C15ull));
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t i = 0; i < img.size(); i += 2) {
        double u1 = (double(ng() >> 11) + 1.0) * (1.0 / 9007199254740993.0);  // (0, 1]
        double u2 = uniform01(ng);
        double r = std::sqrt(-2.0 * std::log(u1));
        double n0 = r * std::cos(two_pi * u2), n1 = r * std::sin(two_pi * u2);
        for (int k = 0; k < 2 && i + k < img.size(); k++) {
            double v = 16.0 + 219.0 * img[i + k] + s->sigma * (k == 0 ? n0 : n1);
            double rv = std::round(v);  // half away from zero
            img[i + k] = rv < 0.0 ? 0.0 : (rv > 255.0 ? 255.0 : rv);
        }
    }
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) out[size_t(y) * stride + x] = uint8_t(img[size_t(y) * W + x]);
    return 0;
}

// n draws of std::mt19937_64(seed) reduced modulo m (the batched configuration's resolution choices).
int ironav_synth_draws(uint64_t seed, int n, int m, int* out) {
    if (n < 0 || m <= 0 || !out) return 3;
    std::mt19937_64 g(seed);
    for (int i = 0; i < n; i++) out[i] = int(g() % uint64_t(m));
    return 0;
}

// The cumulative pan of frame t in quarter samples (for tests that check recovered motion).
int ironav_synth_pan(void* h, int t, int* qx, int* qy) {
    Synth* s = static_cast<Synth*>(h);
    if (!s || t < 0 || t >= int(s->px.size())) return 3;
    *qx = int(std::lround(s->px[t] * 4.0));
    *qy = int(std::lround(s->py[t] * 4.0));
    return 0;
}

}  // extern "C"
