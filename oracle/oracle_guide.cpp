// oracle_guide.cpp -- CPU restatement of the path-guiding network (TEST INFRASTRUCTURE ONLY).
//
// No reference counterpart (the reference has no learned guiding). This is the checker for the
// GPU network: the same architecture written out as plain loops in double precision --
//   inputs (position normalised to the box, normal, direction) -> per input sin/cos(pi 2^(f/2) x),
//   f = 0..11 (216 features), then the 9 raw inputs, zero padding to 256 -> W0 (256x64) -> ReLU ->
//   W1..W4 (64x64, ReLU) -> W5 (64x48; 40 used) -> 8 vMF lobes (mean m/|m|, +z for m = 0, concentration
//   exp(clamp(s, -6, 7)), weight softmax) -- and the KL loss of neural importance sampling
//   (Mueller et al. 2019): L = -(1/B) sum_i min(w_i / mean(w), 20) * log q(d_i | x_i), its gradient by
//   hand-written backpropagation, and mixture sampling (lobe by weight, vMF direction by the
//   inverse CDF of its cosine, Jakob 2012, frame of Duff et al. 2017).
// With `emulate` set, values are rounded to bf16 (round to nearest even) where the GPU stores them
// in bf16: weights, encoded features, hidden activations, the output gradient and the layer deltas.
#include <stdint.h>
#include <string.h>

#include <cmath>
#include <vector>

namespace {

constexpr int kIn = 9, kFreq = 12, kEnc = 256, kEncUsed = 225, kW = 64, kOut = 48, kLobes = 8;
constexpr int kOff[7] = {0, 256 * 64, 256 * 64 + 4096, 256 * 64 + 2 * 4096, 256 * 64 + 3 * 4096, 256 * 64 + 4 * 4096,
                         256 * 64 + 4 * 4096 + 64 * 48};
constexpr double kPi = 3.14159265358979323846;

float bf16(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return x;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

struct Net {
    std::vector<double> W;  // kOff[6] weights (bf16-rounded when emulating)
    bool em;
    double r(double v) const { return em ? (double)bf16((float)v) : v; }
    int K(int l) const { return l == 0 ? kEnc : kW; }
    int N(int l) const { return l == 5 ? kOut : kW; }
    double w(int l, int k, int n) const { return W[kOff[l] + k * N(l) + n]; }
};

Net make_net(const float* params, int emulate) {
    Net net;
    net.em = emulate != 0;
    net.W.resize(kOff[6]);
    for (int i = 0; i < kOff[6]; ++i) net.W[i] = net.em ? (double)bf16(params[i]) : (double)params[i];
    return net;
}

void normalise(const float* raw, const float* lo, const float* hi, double* x) {
    for (int c = 0; c < 3; ++c) {
        const float e = hi[c] - lo[c];
        x[c] = (double)((raw[c] - lo[c]) * (e > 0 ? 1.0f / e : 0.0f));
    }
    for (int c = 3; c < kIn; ++c) x[c] = raw[c];
}

void encode(const Net& net, const double* x, double* e) {
    for (int c = 0; c < kEnc; ++c) {
        double v = 0.0;
        if (c < kIn * 2 * kFreq) {
            const int d = c / (2 * kFreq), j = c % (2 * kFreq), f = j >> 1;
            const double a = kPi * ((double)(float)(x[d] * (double)(float)std::exp2(0.5 * f)));
            v = (j & 1) ? std::cos(a) : std::sin(a);
        } else if (c < kEncUsed) {
            v = x[c - kIn * 2 * kFreq];
        }
        e[c] = net.r(v);
    }
}

// h[0] = encoding (256), h[1..5] = hidden activations (64), out (48)
struct Fwd {
    double h[6][kEnc];
    double out[kOut];
};

void forward(const Net& net, const double* x, Fwd& F) {
    encode(net, x, F.h[0]);
    for (int l = 0; l < 6; ++l) {
        const int K = net.K(l), N = net.N(l);
        for (int n = 0; n < N; ++n) {
            double s = 0.0;
            for (int k = 0; k < K; ++k) s += F.h[l][k] * net.w(l, k, n);
            if (l < 5) F.h[l + 1][n] = net.r(s > 0.0 ? s : 0.0);
            else F.out[n] = s;
        }
    }
}

struct Mix {
    double mu[kLobes][3], kappa[kLobes], pi[kLobes], norm[kLobes];
};

void mixture(const double* o, Mix& M) {
    double mx = -1e300;
    for (int l = 0; l < kLobes; ++l) mx = std::max(mx, o[5 * l + 4]);
    double sum = 0.0;
    for (int l = 0; l < kLobes; ++l) {
        const double n = std::sqrt(o[5 * l] * o[5 * l] + o[5 * l + 1] * o[5 * l + 1] + o[5 * l + 2] * o[5 * l + 2]);
        M.norm[l] = n;
        for (int c = 0; c < 3; ++c) M.mu[l][c] = n > 0.0 ? o[5 * l + c] / n : (c == 2 ? 1.0 : 0.0);
        M.kappa[l] = std::exp(std::min(std::max(o[5 * l + 3], -6.0), 7.0));
        M.pi[l] = std::exp(o[5 * l + 4] - mx);
        sum += M.pi[l];
    }
    for (int l = 0; l < kLobes; ++l) M.pi[l] /= sum;
}

double vmf_log(double kappa, double c) {
    return std::log(kappa / (-std::expm1(-2.0 * kappa))) - std::log(2.0 * kPi) + kappa * (c - 1.0);
}

// -log q(d) and its gradient with respect to the 40 raw outputs, times ws
double record_grad(const double* o, const double* d, double ws, double* g) {
    Mix M;
    mixture(o, M);
    double la[kLobes], cs[kLobes], mx = -1e300;
    for (int l = 0; l < kLobes; ++l) {
        cs[l] = M.mu[l][0] * d[0] + M.mu[l][1] * d[1] + M.mu[l][2] * d[2];
        la[l] = std::log(M.pi[l]) + vmf_log(M.kappa[l], cs[l]);
        mx = std::max(mx, la[l]);
    }
    double s = 0.0;
    for (int l = 0; l < kLobes; ++l) s += std::exp(la[l] - mx);
    const double lq = mx + std::log(s);
    for (int l = 0; l < kLobes; ++l) {
        const double r = std::exp(la[l] - lq), k = M.kappa[l], c = -ws * r;
        g[5 * l + 4] = -ws * (r - M.pi[l]);
        const double sk = o[5 * l + 3];
        g[5 * l + 3] = (sk > -6.0 && sk < 7.0) ? c * k * (1.0 / k - 2.0 / std::expm1(2.0 * k) + cs[l] - 1.0) : 0.0;
        const double f = c * k / std::max(M.norm[l], 1e-3);
        for (int q = 0; q < 3; ++q) g[5 * l + q] = f * (d[q] - cs[l] * M.mu[l][q]);
    }
    for (int q = 40; q < kOut; ++q) g[q] = 0.0;
    return -lq;
}

void onb(const double* n, double* t, double* b) {
    const double sign = std::copysign(1.0, n[2]);
    const double a = -1.0 / (sign + n[2]);
    const double bb = n[0] * n[1] * a;
    t[0] = 1.0 + sign * n[0] * n[0] * a;
    t[1] = sign * bb;
    t[2] = -sign * n[0];
    b[0] = bb;
    b[1] = sign + n[1] * n[1] * a;
    b[2] = -n[1];
}

}  // namespace

extern "C" int oracle_guide_forward(const float* params, const float* inputs, uint64_t n, const float* lo, const float* hi,
                                    int emulate, float* raw48, float* mix40) {
    const Net net = make_net(params, emulate);
    Fwd F;
    for (uint64_t i = 0; i < n; ++i) {
        double x[kIn];
        normalise(inputs + 9 * i, lo, hi, x);
        forward(net, x, F);
        if (raw48)
            for (int c = 0; c < kOut; ++c) raw48[kOut * i + c] = (float)F.out[c];
        if (mix40) {
            Mix M;
            mixture(F.out, M);
            float* m = mix40 + 40 * i;
            for (int l = 0; l < kLobes; ++l) {
                for (int c = 0; c < 3; ++c) m[4 * l + c] = (float)M.mu[l][c];
                m[4 * l + 3] = (float)M.kappa[l];
                m[32 + l] = (float)M.pi[l];
            }
        }
    }
    return 0;
}

// gradient of the mean loss over n records (13 floats each) with respect to the kOff[6] weights
extern "C" int oracle_guide_grad(const float* params, const float* records, uint64_t n, const float* lo, const float* hi,
                                 int emulate, double* grad, double* loss) {
    const Net net = make_net(params, emulate);
    for (int i = 0; i < kOff[6]; ++i) grad[i] = 0.0;
    double wsum = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        const float w = records[13 * i + 12];
        if (w > 0.0f && std::isfinite(w)) wsum += (double)w;
    }
    const double inv_mean = (wsum > 0 && n > 0) ? (double)n / (double)(float)wsum : 0.0;
    const double inv_b = n > 0 ? 1.0 / (double)n : 0.0;
    double L = 0.0;
    Fwd F;
    double delta[6][kW];
    for (uint64_t i = 0; i < n; ++i) {
        const float* rec = records + 13 * i;
        double x[kIn];
        normalise(rec, lo, hi, x);
        forward(net, x, F);
        float wf = rec[12];
        if (!(wf > 0.0f) || !std::isfinite(wf)) wf = 0.0f;
        const double wn = std::min((double)(float)((double)wf * inv_mean), 20.0);
        const double d[3] = {rec[9], rec[10], rec[11]};
        double g[kOut];
        L += wn * record_grad(F.out, d, wn * inv_b, g);
        for (int c = 0; c < kOut; ++c) g[c] = net.r(g[c]);
        // backward: delta_5 from W5, then down to delta_1
        for (int l = 5; l >= 1; --l) {
            const int N = net.N(l);
            const double* up = l == 5 ? g : delta[l + 1];
            for (int k = 0; k < kW; ++k) {
                double s = 0.0;
                for (int nn = 0; nn < N; ++nn) s += up[nn] * net.w(l, k, nn);
                delta[l][k] = net.r(F.h[l][k] > 0.0 ? s : 0.0);
            }
        }
        for (int l = 0; l < 6; ++l) {
            const int K = net.K(l), N = net.N(l);
            const double* up = l == 5 ? g : delta[l + 1];
            double* G = grad + kOff[l];
            for (int k = 0; k < K; ++k) {
                const double hk = F.h[l][k];
                if (hk == 0.0) continue;
                for (int nn = 0; nn < N; ++nn) G[k * N + nn] += hk * up[nn];
            }
        }
    }
    if (loss) *loss = L * inv_b;
    return 0;
}

// mixture (40 floats: 8 x (mu, kappa), 8 weights) at n directions -> density
extern "C" int oracle_vmf_pdf(const float* mix40, const float* dirs, uint64_t n, float* pdf) {
    for (uint64_t i = 0; i < n; ++i) {
        const float* m = mix40 + 40 * i;
        const float* d = dirs + 3 * i;
        double p = 0.0;
        for (int l = 0; l < kLobes; ++l) {
            const double c = m[4 * l] * (double)d[0] + m[4 * l + 1] * (double)d[1] + m[4 * l + 2] * (double)d[2];
            p += m[32 + l] * std::exp(vmf_log(m[4 * l + 3], c));
        }
        pdf[i] = (float)p;
    }
    return 0;
}

// mixture sampling with uniforms u (n x 3: lobe choice, cosine, azimuth) -> directions, density
extern "C" int oracle_vmf_sample(const float* mix40, const float* u, uint64_t n, float* dirs, float* pdf) {
    for (uint64_t i = 0; i < n; ++i) {
        const float* m = mix40 + 40 * i;
        int lobe = kLobes - 1;
        double acc = 0.0;
        for (int l = 0; l < kLobes; ++l) {
            acc += m[32 + l];
            if (u[3 * i] < acc) {
                lobe = l;
                break;
            }
        }
        const double k = m[4 * lobe + 3];
        const double u1 = u[3 * i + 1], u2 = u[3 * i + 2];
        double w = 1.0 + std::log(u1 + (1.0 - u1) * std::exp(-2.0 * k)) / k;
        w = std::min(1.0, std::max(-1.0, w));
        const double s = std::sqrt(std::max(0.0, 1.0 - w * w));
        const double mu[3] = {m[4 * lobe], m[4 * lobe + 1], m[4 * lobe + 2]};
        double t[3], b[3];
        onb(mu, t, b);
        const double ph = 2.0 * kPi * u2;
        for (int c = 0; c < 3; ++c) dirs[3 * i + c] = (float)(w * mu[c] + s * (std::cos(ph) * t[c] + std::sin(ph) * b[c]));
    }
    return oracle_vmf_pdf(mix40, dirs, n, pdf);
}
