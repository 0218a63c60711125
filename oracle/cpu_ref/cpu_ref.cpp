// C++17/OpenMP restatement of the reference's CPU MD step (test
// infrastructure: the timed CPU baseline and the `bench.py --impl reference`
// arm; never part of the product).
//
// The reference (Rust crate `dynamics` 0.2.2) cannot be compiled here, so this
// restates its CPU algorithm for one step, MdState::step
// (src/integrate.rs:72-473), for rigid OPC water plus non-water atoms
// (peptides, ions) with bonded terms and bond-to-H constraints:
//   * neighbour lists: O(N^2) brute force, |min_image(d)|^2 < (rc + skin)^2,
//     half lists mirrored, rows in parallel (src/neighbors.rs:102-281);
//     rebuilt when the max O displacement since the last build reaches
//     skin / 2 (src/neighbors.rs:56-83,159-169);
//   * flat pair list in setup_pairs order (src/non_bonded.rs:541-677);
//   * pair forces: parallel fold with per-thread float64 force arrays and a
//     reduce (src/non_bonded.rs:258-412), pair math of f_nonbonded_cpu
//     (src/non_bonded.rs:950-1057) in float32;
//   * SPME every 2 steps with cached forces (src/lib.rs:1282-1341): order-4
//     B-spline spread, 3D FFT (a mixed-radix FFT written here), influence
//     function, gather, k-space virial; the PME tables are rebuilt every step
//     as regen_pme does (src/integrate.rs:192);
//   * rigid water drift, serial (src/solvent/opc_settle.rs:107-198);
//   * bonds, angles, dihedrals, serial (src/bonded.rs:23-135); the 1-4
//     vacuum Coulomb correction after SPME (src/non_bonded.rs:763-790);
//     lincs_hydrogens + rattle_hydrogens (src/bonded.rs:218-304);
//   * Langevin-middle OU step, serial (src/thermostat.rs:308-362), or
//     velocity Verlet + CSVR (src/thermostat.rs:258-304);
//   * KE (src/thermostat.rs:46-84), pressure (src/barostat.rs:419-431),
//     linear COM removal every 100 steps (src/com_zero.rs:57-81).
//
// Input (binary, little endian): see main().  Output: one JSON line; with a
// third argument, the forces of the first evaluation written to that file
// instead (no steps are run).
#include <omp.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

using cd = std::complex<double>;

namespace {

// ---- constants (src/solvent/mod.rs:58-94, src/lib.rs:196) ----
const float O_MASS = 16.0f, H_MASS = 1.008f, MASS_MOL = 16.0f + 2.0f * 1.008f;
const float O_EP_R = 0.15939833f;
const float CHARGE_UNIT_SCALER = 18.2223f;
const float Q_H = 0.6791f * CHARGE_UNIT_SCALER, Q_EP = -2.0f * Q_H;
const float O_SIGMA = 1.777167268f * (2.0f / 1.122462048309373f), O_EPS = 0.2128008130f;
const float RA = 0.5395199719801114f;
const float C_H = (O_EP_R / RA) / 2.0f, C_O = 1.0f - 2.0f * C_H;
const float KCAL_TO_NATIVE = 418.4f;
const float KB_NATIVE = 0.83144626f;
const double GAS_R = 0.0019872041;
const double BAR = 69476.95457055373;
const float INV_SQRT_PI = 0.5641895835477563f;

struct V3 {
    float x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

struct Box {
    V3 lo, ext;
    V3 min_image(V3 d) const {  // src/barostat.rs:162-170 (round: ties away)
        return {d.x - std::round(d.x / ext.x) * ext.x, d.y - std::round(d.y / ext.y) * ext.y,
                d.z - std::round(d.z / ext.z) * ext.z};
    }
    static float rem_euclid(float a, float b) {
        float r = std::fmod(a, b);
        return r < 0 ? r + std::fabs(b) : r;
    }
    V3 wrap(V3 p) const {  // src/barostat.rs:141-157
        return {rem_euclid(p.x - lo.x, ext.x) + lo.x, rem_euclid(p.y - lo.y, ext.y) + lo.y,
                rem_euclid(p.z - lo.z, ext.z) + lo.z};
    }
    double volume() const { return (double)ext.x * ext.y * ext.z; }
};

struct Water {
    V3 o, h0, h1, m;           // positions
    V3 vo, vh0, vh1;           // velocities
    V3 ao, ah0, ah1;           // accelerations
    V3 fo, fh0, fh1, fm;       // forces
};

struct Pair {  // NonBondedPair (src/non_bonded.rs:219-232)
    uint32_t i, j;
    uint8_t s0, s1;  // water sites 0 O, 1 M, 2 H0, 3 H1; 4 = a non-water atom
    uint8_t lj, coul, scale14;
};

struct Atom {
    V3 p, v, a, f;
    float m, q, sig, eps;
};
struct Bond { uint32_t i, j; float k, r0; };
struct Angle { uint32_t i, j, l; float k, t0; };
struct Dihedral { uint32_t i, j, k, l; float kk, n, ph; };
struct Constraint { uint32_t h, x; float r02, im; };  // heavy, hydrogen

struct Sim {
    Box box;
    std::vector<Water> w;
    std::vector<Atom> at;
    std::vector<uint64_t> excl, p14;  // sorted keys i * 2^32 + j, i < j
    std::vector<Bond> bonds;
    std::vector<Angle> angles;
    std::vector<Dihedral> dih;
    std::vector<Constraint> cons;
    double vir_cons = 0;
    float rc, lj_cutoff, alpha, skin;
    int grid[3];
    int integrator;  // 0 Langevin-middle, 1 VV + CSVR
    float gamma, temp, tau;
    uint64_t step = 0;
    std::vector<Pair> pairs;
    std::vector<V3> o_last, a_last;
    float max_disp2 = 0.f;
    // SPME cache (src/lib.rs:1296-1340)
    std::vector<V3> spme_f;
    std::vector<V3> spme_df14;  // 1-4 vacuum correction of the last SPME step
    double spme_e = 0, spme_w = 0;
    double ke = 0, pe = 0, virial = 0;
    int rebuilds = 0;
    std::mt19937_64 rng{12345};
    std::normal_distribution<float> nd{0.f, 1.f};
};

V3 site_pos(const Water& w, int s) { return s == 0 ? w.o : s == 1 ? w.m : s == 2 ? w.h0 : w.h1; }

inline uint64_t key(uint32_t a, uint32_t b) {
    return a < b ? ((uint64_t)a << 32) | b : ((uint64_t)b << 32) | a;
}
inline bool has(const std::vector<uint64_t>& v, uint64_t k) { return std::binary_search(v.begin(), v.end(), k); }

// ---------------------------------------------------------------- lists --
void build_neighbors(Sim& S) {
    const int n = (int)S.w.size();
    std::vector<V3> o(n);
    for (int i = 0; i < n; ++i) o[i] = S.box.wrap(S.w[i].o);
    const float cs = S.rc + S.skin;
    const float thr = cs * cs;
    std::vector<std::vector<uint32_t>> half(n);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            const V3 d = S.box.min_image(o[i] - o[j]);
            if (d.x * d.x + d.y * d.y + d.z * d.z < thr) half[i].push_back((uint32_t)j);
        }
    }
    // non-water atoms: std-std (i < j) and std-water lists (src/neighbors.rs:180-281)
    const int na = (int)S.at.size();
    std::vector<std::vector<uint32_t>> ss(na), sw(na);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < na; ++i) {
        const V3 pi = S.box.wrap(S.at[i].p);
        for (int j = i + 1; j < na; ++j) {
            const V3 d = S.box.min_image(pi - S.box.wrap(S.at[j].p));
            if (dot(d, d) < thr) ss[i].push_back((uint32_t)j);
        }
        for (int j = 0; j < n; ++j) {
            const V3 d = S.box.min_image(pi - o[j]);
            if (dot(d, d) < thr) sw[i].push_back((uint32_t)j);
        }
    }
    // setup_pairs order: std-std, std-water, water-water (src/non_bonded.rs:541-677);
    // 1-2 / 1-3 pairs are left out, 1-4 pairs flagged
    S.pairs.clear();
    for (int i = 0; i < na; ++i)
        for (uint32_t j : ss[i]) {
            const uint64_t k = key((uint32_t)i, j);
            if (has(S.excl, k)) continue;
            S.pairs.push_back({(uint32_t)i, j, 4, 4, 1, 1, (uint8_t)has(S.p14, k)});
        }
    for (int i = 0; i < na; ++i)
        for (uint32_t j : sw[i])
            for (uint8_t b = 0; b < 4; ++b) S.pairs.push_back({(uint32_t)i, j, 4, b, (uint8_t)(b == 0), (uint8_t)(b != 0), 0});
    for (int i = 0; i < n; ++i)
        for (uint32_t j : half[i])
            for (uint8_t a = 0; a < 4; ++a)
                for (uint8_t b = 0; b < 4; ++b) {
                    const bool lj = a == 0 && b == 0, co = a != 0 && b != 0;
                    if (!(lj || co)) continue;
                    S.pairs.push_back({(uint32_t)i, j, a, b, (uint8_t)lj, (uint8_t)co, 0});
                }
    S.o_last = o;
    S.a_last.resize(na);
    for (int i = 0; i < na; ++i) S.a_last[i] = S.at[i].p;
    S.max_disp2 = 0.f;
    S.rebuilds++;
}

// -------------------------------------------------------- pair forces --
void pair_forces(Sim& S) {
    const int n = (int)S.w.size(), na = (int)S.at.size();
    const size_t nf = 12 * (size_t)n + 3 * (size_t)na;  // waters, then atoms
    const int nt = omp_get_max_threads();
    std::vector<std::vector<double>> acc(nt, std::vector<double>(nf, 0.0));
    std::vector<double> vir(nt, 0.0);
    const float rc = S.rc, a = S.alpha, ljc = S.lj_cutoff;
    const float q[4] = {0.f, Q_EP, Q_H, Q_H};
#pragma omp parallel
    {
        const int t = omp_get_thread_num();
        double* F = acc[t].data();
        double w_acc = 0.0;
#pragma omp for schedule(static)
        for (long long p = 0; p < (long long)S.pairs.size(); ++p) {
            const Pair& pr = S.pairs[p];
            const bool ai = pr.s0 == 4, aj = pr.s1 == 4;
            const V3 pi = ai ? S.at[pr.i].p : site_pos(S.w[pr.i], pr.s0);
            const V3 pj = aj ? S.at[pr.j].p : site_pos(S.w[pr.j], pr.s1);
            const V3 d = S.box.min_image(pi - pj);
            const float r2 = dot(d, d);
            if (r2 < 1e-12f) continue;
            const float r = std::sqrt(r2);
            const float ir = 1.0f / r;
            const V3 dir = d * ir;
            float fm = 0.f;
            float sig = O_SIGMA, eps = O_EPS;
            if (ai || aj) {  // LjTables / combine_lj_params (src/non_bonded.rs:1081-1086)
                const float si = ai ? S.at[pr.i].sig : O_SIGMA, ei = ai ? S.at[pr.i].eps : O_EPS;
                const float sj = aj ? S.at[pr.j].sig : O_SIGMA, ej = aj ? S.at[pr.j].eps : O_EPS;
                sig = 0.5f * (si + sj);
                eps = std::sqrt(ei * ej);
            }
            if (pr.lj && r <= ljc && eps != 0.f) {
                const float sr = sig * ir, sr2 = sr * sr, sr4 = sr2 * sr2, sr6 = sr4 * sr2, sr12 = sr6 * sr6;
                float fl = 24.f * eps * (2.f * sr12 - sr6) * ir;
                if (pr.scale14) fl *= 0.5f;
                fm += fl;
            }
            const float qi = ai ? S.at[pr.i].q : q[pr.s0], qj = aj ? S.at[pr.j].q : q[pr.s1];
            if (pr.coul && r < rc && qi * qj != 0.f) {
                const float ar = a * r;
                float fc = qi * qj * (std::erfc(ar) * ir * ir + 2.f * a * std::exp(-ar * ar) * INV_SQRT_PI * ir);
                if (pr.scale14) fc *= 1.0f / 1.2f;
                fm += fc;
            }
            const V3 f = dir * fm;
            w_acc += (double)dot(d, f);
            double* fi = ai ? F + 12 * (size_t)n + 3 * (size_t)pr.i : F + 12 * (size_t)pr.i + 3 * pr.s0;
            double* fj = aj ? F + 12 * (size_t)n + 3 * (size_t)pr.j : F + 12 * (size_t)pr.j + 3 * pr.s1;
            fi[0] += f.x; fi[1] += f.y; fi[2] += f.z;
            fj[0] -= f.x; fj[1] -= f.y; fj[2] -= f.z;
        }
        vir[t] = w_acc;
    }
    // reduce (src/non_bonded.rs:373-411)
    std::vector<double> tot(nf, 0.0);
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)nf; ++k) {
        double s = 0;
        for (int t = 0; t < nt; ++t) s += acc[t][k];
        tot[k] = s;
    }
    S.virial = 0;
    for (int t = 0; t < nt; ++t) S.virial += vir[t];
    for (int i = 0; i < n; ++i) {
        Water& w = S.w[i];
        const double* f = &tot[12 * (size_t)i];
        w.fo = w.fo + V3{(float)f[0], (float)f[1], (float)f[2]};
        w.fm = w.fm + V3{(float)f[3], (float)f[4], (float)f[5]};
        w.fh0 = w.fh0 + V3{(float)f[6], (float)f[7], (float)f[8]};
        w.fh1 = w.fh1 + V3{(float)f[9], (float)f[10], (float)f[11]};
    }
    for (int i = 0; i < na; ++i) {
        const double* f = &tot[12 * (size_t)n + 3 * (size_t)i];
        S.at[i].f = S.at[i].f + V3{(float)f[0], (float)f[1], (float)f[2]};
    }
}

// ------------------------------------------------------------- bonded --
// apply_bonded_forces (src/bonded.rs:23-135), f_bond_stretching /
// f_angle_bending / f_dihedral (src/bonded_forces.rs:11-178), serial
void bonded_forces(Sim& S) {
    auto& A = S.at;
    double vir = 0;
    for (const Bond& b : S.bonds) {
        const V3 d = S.box.min_image(A[b.j].p - A[b.i].p);
        const float r = std::sqrt(dot(d, d));
        const V3 f = d * (2.f * b.k * (r - b.r0) / std::max(r, 1e-8f));
        A[b.i].f = A[b.i].f + f;
        A[b.j].f = A[b.j].f - f;
        vir += dot(d, f);
    }
    for (const Angle& g : S.angles) {
        const V3 v01 = S.box.min_image(A[g.i].p - A[g.j].p), v21 = S.box.min_image(A[g.l].p - A[g.j].p);
        const float l01 = std::sqrt(dot(v01, v01)), l21 = std::sqrt(dot(v21, v21));
        if (l01 < 1e-4f || l21 < 1e-4f) continue;
        const V3 u01 = v01 * (1.f / l01), u21 = v21 * (1.f / l21);
        const float ct = std::min(1.f, std::max(-1.f, dot(u01, u21)));
        const float st = std::max(std::sqrt(1.f - ct * ct), 1e-8f);
        const float de = 2.f * g.k * (std::acos(ct) - g.t0);
        const V3 f0 = (u01 * ct - u21) * (-de / (l01 * st));
        const V3 f2 = (u21 * ct - u01) * (-de / (l21 * st));
        A[g.i].f = A[g.i].f + f0;
        A[g.l].f = A[g.l].f + f2;
        A[g.j].f = A[g.j].f - f0 - f2;
        vir += dot(v01, f0) + dot(v21, f2);
    }
    for (const Dihedral& q : S.dih) {
        const V3 b1 = S.box.min_image(A[q.j].p - A[q.i].p), b2 = S.box.min_image(A[q.k].p - A[q.j].p),
                 b3 = S.box.min_image(A[q.l].p - A[q.k].p);
        const V3 n1 = cross(b1, b2), n2 = cross(b2, b3);
        const float n1s = dot(n1, n1), n2s = dot(n2, n2), b2s = dot(b2, b2), b2n = std::sqrt(b2s);
        if (n1s < 1e-6f || n2s < 1e-6f || b2n < 1e-6f) continue;
        const float phi = std::atan2(dot(cross(n1, n2), b2) / b2n, dot(n1, n2));
        const float dv = -q.kk * q.n * std::sin(q.n * phi - q.ph);
        const V3 g0 = n1 * (-b2n / n1s), g3 = n2 * (b2n / n2s);
        const float ta = dot(b1, b2) / b2s, tb = dot(b3, b2) / b2s;
        const V3 g1 = g0 * (-1.f - ta) + g3 * tb, g2 = g3 * (-1.f - tb) + g0 * ta;
        A[q.i].f = A[q.i].f + g0 * (-dv); A[q.j].f = A[q.j].f + g1 * (-dv);
        A[q.k].f = A[q.k].f + g2 * (-dv); A[q.l].f = A[q.l].f + g3 * (-dv);
        vir += dot(b1 * -1.f, g0 * (-dv)) + dot(b2, g2 * (-dv)) + dot(b2 + b3, g3 * (-dv));
    }
    S.virial += vir;
}

// ---------------------------------------------------------------- FFT --
// Mixed-radix decimation-in-time Cooley-Tukey with a precomputed twiddle
// table (w[k] = exp(-+2 pi i k / n)); lines are gathered into scratch.
struct FftPlan {
    int n = 0;
    std::vector<cd> wf, wi;
    explicit FftPlan(int n_) : n(n_), wf(n_), wi(n_) {
        for (int k = 0; k < n; ++k) {
            const double a = 2.0 * M_PI * k / n;
            wf[k] = cd(std::cos(a), -std::sin(a));
            wi[k] = cd(std::cos(a), std::sin(a));
        }
    }
};

void fft_rec(const cd* x, cd* y, int N, int s, const cd* w, int n, cd* scratch) {
    if (N == 1) { y[0] = x[0]; return; }
    int p = 2;
    while (N % p) ++p;
    const int m = N / p;
    cd* sub = scratch;
    for (int r = 0; r < p; ++r) fft_rec(x + (size_t)r * s, sub + (size_t)r * m, m, s * p, w, n, scratch + N);
    const int step = n / N;
    for (int k = 0; k < m; ++k)
        for (int q = 0; q < p; ++q) {
            cd acc = sub[k];
            for (int r = 1; r < p; ++r) acc += sub[(size_t)r * m + k] * w[((size_t)r * (k + q * m) * step) % n];
            y[k + q * m] = acc;
        }
}

void fft1d(cd* a, int n, int stride, const FftPlan& pl, bool inv, std::vector<cd>& tmp) {
    cd* in = tmp.data();
    cd* out = in + n;
    cd* scr = out + n;
    for (int i = 0; i < n; ++i) in[i] = a[(size_t)i * stride];
    fft_rec(in, out, n, 1, inv ? pl.wi.data() : pl.wf.data(), n, scr);
    for (int i = 0; i < n; ++i) a[(size_t)i * stride] = out[i];
}

void fft3d(std::vector<cd>& g, const int* K, bool inv) {
    const int K0 = K[0], K1 = K[1], K2 = K[2];
    const FftPlan p0(K0), p1(K1), p2(K2);
    const int kmax = std::max(K0, std::max(K1, K2));
#pragma omp parallel
    {
        std::vector<cd> tmp(4 * (size_t)kmax + 16);
#pragma omp for
        for (int xy = 0; xy < K0 * K1; ++xy) fft1d(&g[(size_t)xy * K2], K2, 1, p2, inv, tmp);
#pragma omp for
        for (int xz = 0; xz < K0 * K2; ++xz) {
            const int x = xz / K2, z = xz % K2;
            fft1d(&g[(size_t)x * K1 * K2 + z], K1, K2, p1, inv, tmp);
        }
#pragma omp for
        for (int yz = 0; yz < K1 * K2; ++yz) fft1d(&g[yz], K0, K1 * K2, p0, inv, tmp);
    }
}

// --------------------------------------------------------------- SPME --
void bspline4(double w, double* th, double* dth) {
    const double w2 = w * w, w3 = w2 * w, om = 1 - w;
    th[0] = om * om * om / 6; th[1] = (3 * w3 - 6 * w2 + 4) / 6;
    th[2] = (-3 * w3 + 3 * w2 + 3 * w + 1) / 6; th[3] = w3 / 6;
    dth[0] = -0.5 * om * om; dth[1] = 1.5 * w2 - 2 * w; dth[2] = -1.5 * w2 + w + 0.5; dth[3] = 0.5 * w2;
}

void spme(Sim& S) {
    const int* K = S.grid;
    const size_t ng = (size_t)K[0] * K[1] * K[2];
    // regen_pme: influence-function tables rebuilt (src/integrate.rs:192)
    std::vector<double> bm[3];
    for (int a = 0; a < 3; ++a) {
        bm[a].resize(K[a]);
        const double mv[3] = {1.0 / 6, 4.0 / 6, 1.0 / 6};
        for (int m = 0; m < K[a]; ++m) {
            double re = 0, im = 0;
            for (int k = 0; k < 3; ++k) { re += mv[k] * cos(2 * M_PI * m * k / K[a]); im += mv[k] * sin(2 * M_PI * m * k / K[a]); }
            bm[a][m] = 1.0 / (re * re + im * im);
        }
    }
    // pack_pme_pos_q (src/non_bonded.rs:800-826): M, H0, H1 per water,
    // then the atoms
    const int n = (int)S.w.size(), na = (int)S.at.size();
    const int nq = 3 * n + na;
    std::vector<V3> pos(nq);
    std::vector<float> q(nq);
    for (int i = 0; i < n; ++i) {
        pos[3 * i] = S.box.wrap(S.w[i].m); q[3 * i] = Q_EP;
        pos[3 * i + 1] = S.box.wrap(S.w[i].h0); q[3 * i + 1] = Q_H;
        pos[3 * i + 2] = S.box.wrap(S.w[i].h1); q[3 * i + 2] = Q_H;
    }
    for (int i = 0; i < na; ++i) { pos[3 * n + i] = S.box.wrap(S.at[i].p); q[3 * n + i] = S.at[i].q; }
    std::vector<cd> grid(ng, 0.0);
    std::vector<int> base(3 * (size_t)nq);
    std::vector<double> th(12 * (size_t)nq), dth(12 * (size_t)nq);
    const double ext[3] = {S.box.ext.x, S.box.ext.y, S.box.ext.z};
    const double lo[3] = {S.box.lo.x, S.box.lo.y, S.box.lo.z};
    for (int i = 0; i < nq; ++i) {
        const double p[3] = {pos[i].x, pos[i].y, pos[i].z};
        for (int a = 0; a < 3; ++a) {
            double u = (p[a] - lo[a]) / ext[a] * K[a];
            u = std::fmod(u, (double)K[a]);
            if (u < 0) u += K[a];
            const int b = (int)std::floor(u);
            base[3 * i + a] = b;
            bspline4(u - b, &th[12 * (size_t)i + 4 * a], &dth[12 * (size_t)i + 4 * a]);
        }
        for (int a = 0; a < 4; ++a) {
            const int x = ((base[3 * i] - 3 + a) % K[0] + K[0]) % K[0];
            for (int b = 0; b < 4; ++b) {
                const int y = ((base[3 * i + 1] - 3 + b) % K[1] + K[1]) % K[1];
                for (int c = 0; c < 4; ++c) {
                    const int z = ((base[3 * i + 2] - 3 + c) % K[2] + K[2]) % K[2];
                    grid[((size_t)x * K[1] + y) * K[2] + z] +=
                        q[i] * th[12 * (size_t)i + a] * th[12 * (size_t)i + 4 + b] * th[12 * (size_t)i + 8 + c];
                }
            }
        }
    }
    fft3d(grid, K, false);
    const double vol = S.box.volume(), pa2 = M_PI * M_PI / ((double)S.alpha * S.alpha);
    double e = 0, w = 0;
#pragma omp parallel for reduction(+ : e, w)
    for (long long idx = 0; idx < (long long)ng; ++idx) {
        const int z = (int)(idx % K[2]), y = (int)((idx / K[2]) % K[1]), x = (int)(idx / ((size_t)K[1] * K[2]));
        const int mx = x <= K[0] / 2 ? x : x - K[0], my = y <= K[1] / 2 ? y : y - K[1],
                  mz = z <= K[2] / 2 ? z : z - K[2];
        const double fx = mx / ext[0], fy = my / ext[1], fz = mz / ext[2];
        const double m2 = fx * fx + fy * fy + fz * fz;
        double g = 0;
        if (m2 > 0) {
            g = bm[0][x] * bm[1][y] * bm[2][z] * std::exp(-pa2 * m2) / (M_PI * vol * m2);
            const double em = 0.5 * g * std::norm(grid[idx]);
            e += em;
            w += em * (1.0 - 2.0 * pa2 * m2);
        }
        grid[idx] *= g;
    }
    fft3d(grid, K, true);
    S.spme_f.assign(nq, V3{0, 0, 0});
#pragma omp parallel for
    for (int i = 0; i < nq; ++i) {
        double g[3] = {0, 0, 0};
        for (int a = 0; a < 4; ++a) {
            const int x = ((base[3 * i] - 3 + a) % K[0] + K[0]) % K[0];
            for (int b = 0; b < 4; ++b) {
                const int y = ((base[3 * i + 1] - 3 + b) % K[1] + K[1]) % K[1];
                for (int c = 0; c < 4; ++c) {
                    const int z = ((base[3 * i + 2] - 3 + c) % K[2] + K[2]) % K[2];
                    const double ph = grid[((size_t)x * K[1] + y) * K[2] + z].real();
                    const double* t = &th[12 * (size_t)i];
                    const double* dt = &dth[12 * (size_t)i];
                    g[0] += dt[a] * t[4 + b] * t[8 + c] * ph;
                    g[1] += t[a] * dt[4 + b] * t[8 + c] * ph;
                    g[2] += t[a] * t[4 + b] * dt[8 + c] * ph;
                }
            }
        }
        S.spme_f[i] = V3{(float)(-q[i] * K[0] / ext[0] * g[0]), (float)(-q[i] * K[1] / ext[1] * g[1]),
                         (float)(-q[i] * K[2] / ext[2] * g[2])};
    }
    double qs = 0;
    for (int i = 0; i < nq; ++i) qs += (double)q[i] * q[i];
    S.spme_e = e - S.alpha / std::sqrt(M_PI) * qs;
    S.spme_w = w;
    // 1-4 vacuum Coulomb correction (src/non_bonded.rs:763-790): applied
    // on the SPME steps only -- its forces are not part of the cached
    // reciprocal forces (src/lib.rs:1296-1340), its virial is
    S.spme_df14.assign(na, V3{0, 0, 0});
    for (const uint64_t k : S.p14) {
        const uint32_t i = (uint32_t)(k >> 32), j = (uint32_t)(k & 0xFFFFFFFFu);
        const V3 d = S.box.min_image(S.at[i].p - S.at[j].p);
        const float r = std::sqrt(dot(d, d));
        if (r < 1e-6f) continue;
        const V3 df = d * (S.at[i].q * S.at[j].q / (r * r * r) * (1.0f / 1.2f - 1.0f));
        S.spme_df14[i] = S.spme_df14[i] + df;
        S.spme_df14[j] = S.spme_df14[j] - df;
    }
}

// -------------------------------------------------------- rigid water --
V3 rodrigues(V3 r, V3 om, float dt) {
    const V3 od = om * dt;
    const float th = std::sqrt(dot(od, od));
    if (th < 1e-12f) {
        const V3 wxr = cross(od, r);
        return r + wxr + cross(od, wxr) * 0.5f;
    }
    const V3 n = od * (1.0f / th);
    const float c = std::cos(th), s = std::sin(th);
    return r * c + cross(n, r) * s + n * (dot(n, r) * (1.0f - c));
}

void rigid(Water& m, float dt, const Box& b) {  // src/solvent/opc_settle.rs:107-198
    const V3 o = m.o;
    const V3 h0 = o + b.min_image(m.h0 - o), h1 = o + b.min_image(m.h1 - o);
    const V3 rc = (o * O_MASS + h0 * H_MASS + h1 * H_MASS) * (1.0f / MASS_MOL);
    const V3 vc = (m.vo * O_MASS + m.vh0 * H_MASS + m.vh1 * H_MASS) * (1.0f / MASS_MOL);
    const V3 rO = o - rc, rH0 = h0 - rc, rH1 = h1 - rc;
    const V3 uO = m.vo - vc, uH0 = m.vh0 - vc, uH1 = m.vh1 - vc;
    const V3 L = cross(rO, uO) * O_MASS + cross(rH0, uH0) * H_MASS + cross(rH1, uH1) * H_MASS;
    float I[6] = {0, 0, 0, 0, 0, 0};
    const V3 rs[3] = {rO, rH0, rH1};
    const float ms[3] = {O_MASS, H_MASS, H_MASS};
    for (int k = 0; k < 3; ++k) {
        const V3 r = rs[k];
        const float r2 = dot(r, r), mm = ms[k];
        I[0] += mm * (r2 - r.x * r.x); I[1] += mm * (r2 - r.y * r.y); I[2] += mm * (r2 - r.z * r.z);
        I[3] += -mm * r.x * r.y; I[4] += -mm * r.x * r.z; I[5] += -mm * r.y * r.z;
    }
    const float ixx = I[0], iyy = I[1], izz = I[2], ixy = I[3], ixz = I[4], iyz = I[5];
    const float det = ixx * (iyy * izz - iyz * iyz) - ixy * (ixy * izz - iyz * ixz) + ixz * (ixy * iyz - iyy * ixz);
    V3 w{0, 0, 0};
    if (std::fabs(det) >= 1e-12f) {
        const float id = 1.0f / det;
        const float i00 = (iyy * izz - iyz * iyz) * id, i01 = (ixz * iyz - ixy * izz) * id;
        const float i02 = (ixy * iyz - ixz * iyy) * id, i11 = (ixx * izz - ixz * ixz) * id;
        const float i12 = (ixz * ixy - ixx * iyz) * id, i22 = (ixx * iyy - ixy * ixy) * id;
        w = {i00 * L.x + i01 * L.y + i02 * L.z, i01 * L.x + i11 * L.y + i12 * L.z, i02 * L.x + i12 * L.y + i22 * L.z};
    }
    const V3 dl = vc * dt;
    const V3 rO2 = rodrigues(rO, w, dt), rH02 = rodrigues(rH0, w, dt), rH12 = rodrigues(rH1, w, dt);
    m.o = b.wrap(rc + dl + rO2);
    m.h0 = m.o + b.min_image(rc + dl + rH02 - m.o);
    m.h1 = m.o + b.min_image(rc + dl + rH12 - m.o);
    m.vo = vc + cross(w, rO2); m.vh0 = vc + cross(w, rH02); m.vh1 = vc + cross(w, rH12);
    const V3 bis = (m.h0 - m.o) + (m.h1 - m.o);
    m.m = m.o + bis * (O_EP_R / std::sqrt(dot(bis, bis)));
}

double kinetic(const Sim& S) {  // src/thermostat.rs:46-64
    double k = 0;
    for (const Water& w : S.w)
        k += (double)(O_MASS * dot(w.vo, w.vo)) + (double)(H_MASS * dot(w.vh0, w.vh0)) + (double)(H_MASS * dot(w.vh1, w.vh1));
    for (const Atom& a : S.at) k += (double)(a.m * dot(a.v, a.v));
    return k * 0.5 / KCAL_TO_NATIVE;
}

double kinetic_trans(const Sim& S) {
    double k = 0;
    for (const Atom& a : S.at) k += (double)(a.m * dot(a.v, a.v));
    for (const Water& w : S.w) {
        const V3 vc = (w.vo * O_MASS + w.vh0 * H_MASS + w.vh1 * H_MASS) * (1.0f / MASS_MOL);
        k += (double)(MASS_MOL * dot(vc, vc));
    }
    return k * 0.5 / KCAL_TO_NATIVE;
}

void all_forces(Sim& S) {
    for (Water& w : S.w) w.fo = w.fh0 = w.fh1 = w.fm = V3{0, 0, 0};
    for (Atom& a : S.at) a.f = V3{0, 0, 0};
    pair_forces(S);
    bonded_forces(S);
    const bool spme_step = S.step % 2 == 0;  // SPME_RATIO (src/lib.rs:208)
    if (spme_step) spme(S);
    const size_t n = S.w.size();
    for (size_t i = 0; i < n; ++i) {
        S.w[i].fm = S.w[i].fm + S.spme_f[3 * i];
        S.w[i].fh0 = S.w[i].fh0 + S.spme_f[3 * i + 1];
        S.w[i].fh1 = S.w[i].fh1 + S.spme_f[3 * i + 2];
    }
    for (size_t i = 0; i < S.at.size(); ++i) {
        S.at[i].f = S.at[i].f + S.spme_f[3 * n + i];
        if (spme_step) S.at[i].f = S.at[i].f + S.spme_df14[i];
    }
    S.pe = S.spme_e;
}

// lincs_hydrogens (src/bonded.rs:218-284), order 4, iter 1, sequential
void lincs(Sim& S, float dt) {
    if (S.cons.empty()) return;
    std::vector<V3> x0(S.at.size());
    for (size_t i = 0; i < S.at.size(); ++i) x0[i] = S.at[i].p;
    for (int o = 0; o < 4; ++o)
        for (const Constraint& c : S.cons) {
            Atom &ai = S.at[c.h], &aj = S.at[c.x];
            const V3 d = aj.p - ai.p;
            const float dl = std::max(std::sqrt(dot(d, d)), 1.1920929e-7f);
            const V3 b = d * (1.f / dl);
            const V3 corr = b * ((std::sqrt(c.r02) - dot(b, d)) / c.im);
            ai.p = ai.p - corr * (1.f / ai.m);
            aj.p = aj.p + corr * (1.f / aj.m);
        }
    for (const Constraint& c : S.cons) {
        Atom &ai = S.at[c.h], &aj = S.at[c.x];
        const V3 d = aj.p - ai.p;
        const float d2 = dot(d, d);
        const V3 corr = d * ((d2 - c.r02) / (2.f * c.im * std::max(d2, 1e-8f)));
        ai.p = ai.p + corr * (1.f / ai.m);
        aj.p = aj.p - corr * (1.f / aj.m);
    }
    const float inv = 1.f / (dt * dt);
    for (const Constraint& c : S.cons)
        S.vir_cons += dot(S.box.min_image(S.at[c.x].p - S.at[c.h].p), (S.at[c.h].p - x0[c.h]) * (S.at[c.h].m * inv));
}

void rattle(Sim& S) {  // rattle_hydrogens (src/bonded.rs:288-304)
    for (const Constraint& c : S.cons) {
        Atom &ai = S.at[c.h], &aj = S.at[c.x];
        const V3 r = aj.p - ai.p;
        const V3 corr = r * (dot(aj.v - ai.v, r) / (c.im * std::max(dot(r, r), 1e-8f)));
        ai.v = ai.v + corr * (1.f / ai.m);
        aj.v = aj.v - corr * (1.f / aj.m);
    }
}

void kick_calc_accel(Sim& S, float dt) {  // src/integrate.rs:515-562
    for (Water& w : S.w) {
        w.fo = w.fo + w.fm * C_O; w.fh0 = w.fh0 + w.fm * C_H; w.fh1 = w.fh1 + w.fm * C_H; w.fm = V3{0, 0, 0};
        w.ao = w.fo * (KCAL_TO_NATIVE / O_MASS); w.ah0 = w.fh0 * (KCAL_TO_NATIVE / H_MASS); w.ah1 = w.fh1 * (KCAL_TO_NATIVE / H_MASS);
        w.vo = w.vo + w.ao * dt; w.vh0 = w.vh0 + w.ah0 * dt; w.vh1 = w.vh1 + w.ah1 * dt;
    }
    for (Atom& a : S.at) {
        a.a = a.f * (KCAL_TO_NATIVE / a.m);
        const float a2 = dot(a.a, a.a);
        if (a2 > 1e10f) a.a = a.a * (1e5f / std::sqrt(a2));  // MAX_ACCEL (src/integrate.rs:26-27)
        a.v = a.v + a.a * dt;
    }
    rattle(S);
    S.ke = kinetic(S);
}

void step(Sim& S, float dt) {
    const float hdt = 0.5f * dt;
    if (S.integrator == 0) {
        S.vir_cons = 0;
        for (Water& w : S.w) {  // kick_and_drift(dt/2, dt/2)
            w.vo = w.vo + w.ao * hdt; w.vh0 = w.vh0 + w.ah0 * hdt; w.vh1 = w.vh1 + w.ah1 * hdt;
            rigid(w, hdt, S.box);
        }
        for (Atom& a : S.at) { a.v = a.v + a.a * hdt; a.p = a.p + a.v * hdt; }
        lincs(S, hdt);
        rattle(S);
        S.ke = kinetic(S);
        // apply_langevin_thermostat (src/thermostat.rs:308-362), serial
        const float c = std::exp(-S.gamma * dt);
        const float num = KB_NATIVE * S.temp * std::max(1.f - c * c, 0.f);
        const float so = std::sqrt(num / O_MASS), sh = std::sqrt(num / H_MASS);
        for (Water& w : S.w) {
            w.vo = w.vo * c + V3{S.nd(S.rng), S.nd(S.rng), S.nd(S.rng)} * so;
            w.vh0 = w.vh0 * c + V3{S.nd(S.rng), S.nd(S.rng), S.nd(S.rng)} * sh;
            w.vh1 = w.vh1 * c + V3{S.nd(S.rng), S.nd(S.rng), S.nd(S.rng)} * sh;
        }
        for (Atom& a : S.at) a.v = a.v * c + V3{S.nd(S.rng), S.nd(S.rng), S.nd(S.rng)} * std::sqrt(num / a.m);
        rattle(S);
        S.ke = kinetic(S);
        for (Water& w : S.w) rigid(w, hdt, S.box);  // drift(dt/2)
        for (Atom& a : S.at) a.p = a.p + a.v * hdt;
        { const double keep = S.vir_cons; lincs(S, hdt); S.vir_cons = keep; }
        all_forces(S);
        (void)((2.0 * kinetic_trans(S) + S.virial + S.spme_w) / (3.0 * S.box.volume()) * BAR);
        kick_calc_accel(S, hdt);
    } else {
        S.vir_cons = 0;
        for (Water& w : S.w) {  // kick_and_drift(dt/2, dt)
            w.vo = w.vo + w.ao * hdt; w.vh0 = w.vh0 + w.ah0 * hdt; w.vh1 = w.vh1 + w.ah1 * hdt;
            rigid(w, dt, S.box);
        }
        for (Atom& a : S.at) { a.v = a.v + a.a * hdt; a.p = a.p + a.v * dt; }
        lincs(S, hdt);
        rattle(S);
        S.ke = kinetic(S);
        all_forces(S);
        (void)((2.0 * kinetic_trans(S) + S.virial + S.spme_w) / (3.0 * S.box.volume()) * BAR);
        kick_calc_accel(S, hdt);
        // CSVR (src/thermostat.rs:258-304)
        const double dof = 6.0 * S.w.size() + 3.0 * S.at.size() - (double)S.cons.size() - 3.0;
        const double ke = kinetic(S);
        const double c = std::exp(-dt / S.tau);
        std::normal_distribution<double> nd(0, 1);
        std::chi_squared_distribution<double> chi(dof - 1.0);
        const double r = nd(S.rng), x = chi(S.rng);
        const double kt = 0.5 * dof * GAS_R * S.temp;
        double kp = ke * c + kt * (1 - c) * ((x + r * r) / dof) + 2 * r * std::sqrt(c * (1 - c) * ke * kt / dof);
        const float lam = (float)std::sqrt(std::max(kp, 1e-20) / ke);
        for (Water& w : S.w) { w.vo = w.vo * lam; w.vh0 = w.vh0 * lam; w.vh1 = w.vh1 * lam; }
        for (Atom& a : S.at) a.v = a.v * lam;
        S.ke = kinetic(S);
    }
    S.step++;
    if (S.step % 100 == 0) {  // zero_linear_momentum (src/com_zero.rs:57-81)
        double p[3] = {0, 0, 0}, m = 0;
        for (const Water& w : S.w) {
            const V3 q = w.vo * O_MASS + w.vh0 * H_MASS + w.vh1 * H_MASS;
            p[0] += q.x; p[1] += q.y; p[2] += q.z; m += MASS_MOL;
        }
        for (const Atom& a : S.at) { p[0] += a.m * a.v.x; p[1] += a.m * a.v.y; p[2] += a.m * a.v.z; m += a.m; }
        const V3 vc{(float)(p[0] / m), (float)(p[1] / m), (float)(p[2] / m)};
        for (Water& w : S.w) { w.vo = w.vo - vc; w.vh0 = w.vh0 - vc; w.vh1 = w.vh1 - vc; }
        for (Atom& a : S.at) a.v = a.v - vc;
    }
    // update_max_displacement_since_rebuild + build_neighbors_if_needed
    for (size_t i = 0; i < S.w.size(); ++i) {
        const V3 d = S.box.min_image(S.w[i].o - S.o_last[i]);
        S.max_disp2 = std::max(S.max_disp2, dot(d, d));
    }
    for (size_t i = 0; i < S.at.size(); ++i) {
        const V3 d = S.at[i].p - S.a_last[i];
        S.max_disp2 = std::max(S.max_disp2, dot(d, d));
    }
    if (S.max_disp2 >= (S.skin * 0.5f) * (S.skin * 0.5f)) build_neighbors(S);
}

}  // namespace

// Input layout: int32 n_water, int32 integrator, int32 steps, int32 warmup,
// float lo[3], float hi[3], float rc, float lj_cutoff, float alpha, float skin,
// int32 grid[3], float dt, float gamma, float temp, float tau,
// float water_pos[n*9], float water_vel[n*9].
int main(int argc, char** argv) {
    if (argc < 2) { std::fprintf(stderr, "usage: cpu_ref input.bin\n"); return 2; }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    int32_t hdr[4];
    float bx[6], par[4], dyn[4];
    int32_t grid[3];
    float dt;
    if (std::fread(hdr, 4, 4, f) != 4 || std::fread(bx, 4, 6, f) != 6 || std::fread(par, 4, 4, f) != 4 ||
        std::fread(grid, 4, 3, f) != 3 || std::fread(&dt, 4, 1, f) != 1 || std::fread(dyn, 4, 3, f) != 3) {
        std::fprintf(stderr, "short header\n");
        return 2;
    }
    Sim S;
    const int n = hdr[0];
    S.integrator = hdr[1];
    const int steps = hdr[2], warmup = hdr[3];
    S.box.lo = {bx[0], bx[1], bx[2]};
    S.box.ext = {bx[3] - bx[0], bx[4] - bx[1], bx[5] - bx[2]};
    S.rc = par[0]; S.lj_cutoff = par[1]; S.alpha = par[2]; S.skin = par[3];
    for (int k = 0; k < 3; ++k) S.grid[k] = grid[k];
    S.gamma = dyn[0]; S.temp = dyn[1]; S.tau = dyn[2];
    std::vector<float> wp(9 * (size_t)n), wv(9 * (size_t)n);
    if (std::fread(wp.data(), 4, wp.size(), f) != wp.size() || std::fread(wv.data(), 4, wv.size(), f) != wv.size()) {
        std::fprintf(stderr, "short body\n");
        return 2;
    }
    // optional tail: int32 n_atoms; pos[3n], vel[3n], mass, q, sigma, eps [n];
    // int32 n + pairs for exclusions and 1-4; int32 n + (i, j) + (k, r0)
    // bonds; int32 n + (i, j, k) + (k, theta0) angles; int32 n + (i, j, k, l)
    // + (k, n, phase) dihedrals; int32 n + (i, j) + r0 constraints
    int32_t na = 0;
    if (std::fread(&na, 4, 1, f) == 1 && na > 0) {
        std::vector<float> ap(3 * (size_t)na), av(3 * (size_t)na), am(na), aq(na), as(na), ae(na);
        bool ok = std::fread(ap.data(), 4, ap.size(), f) == ap.size() && std::fread(av.data(), 4, av.size(), f) == av.size() &&
                  std::fread(am.data(), 4, na, f) == (size_t)na && std::fread(aq.data(), 4, na, f) == (size_t)na &&
                  std::fread(as.data(), 4, na, f) == (size_t)na && std::fread(ae.data(), 4, na, f) == (size_t)na;
        if (!ok) { std::fprintf(stderr, "short atoms\n"); return 2; }
        S.at.resize(na);
        for (int i = 0; i < na; ++i) {
            Atom& a = S.at[i];
            a.p = {ap[3 * i], ap[3 * i + 1], ap[3 * i + 2]};
            a.v = {av[3 * i], av[3 * i + 1], av[3 * i + 2]};
            a.a = a.f = V3{0, 0, 0};
            a.m = am[i]; a.q = aq[i]; a.sig = as[i]; a.eps = ae[i];
        }
        auto rd_u = [&](std::vector<uint32_t>& v, size_t k) { v.resize(k); return std::fread(v.data(), 4, k, f) == k; };
        auto rd_f = [&](std::vector<float>& v, size_t k) { v.resize(k); return std::fread(v.data(), 4, k, f) == k; };
        int32_t m = 0;
        std::vector<uint32_t> u;
        std::vector<float> fl;
        for (int pass = 0; pass < 2; ++pass) {
            if (std::fread(&m, 4, 1, f) != 1 || !rd_u(u, 2 * (size_t)m)) { std::fprintf(stderr, "short pairs\n"); return 2; }
            std::vector<uint64_t>& dst = pass == 0 ? S.excl : S.p14;
            for (int k = 0; k < m; ++k) dst.push_back(key(u[2 * k], u[2 * k + 1]));
            std::sort(dst.begin(), dst.end());
        }
        if (std::fread(&m, 4, 1, f) != 1 || !rd_u(u, 2 * (size_t)m) || !rd_f(fl, 2 * (size_t)m)) return 2;
        for (int k = 0; k < m; ++k) S.bonds.push_back({u[2 * k], u[2 * k + 1], fl[2 * k], fl[2 * k + 1]});
        if (std::fread(&m, 4, 1, f) != 1 || !rd_u(u, 3 * (size_t)m) || !rd_f(fl, 2 * (size_t)m)) return 2;
        for (int k = 0; k < m; ++k) S.angles.push_back({u[3 * k], u[3 * k + 1], u[3 * k + 2], fl[2 * k], fl[2 * k + 1]});
        if (std::fread(&m, 4, 1, f) != 1 || !rd_u(u, 4 * (size_t)m) || !rd_f(fl, 3 * (size_t)m)) return 2;
        for (int k = 0; k < m; ++k)
            S.dih.push_back({u[4 * k], u[4 * k + 1], u[4 * k + 2], u[4 * k + 3], fl[3 * k], fl[3 * k + 1], fl[3 * k + 2]});
        if (std::fread(&m, 4, 1, f) != 1 || !rd_u(u, 2 * (size_t)m) || !rd_f(fl, (size_t)m)) return 2;
        for (int k = 0; k < m; ++k) {
            uint32_t h = u[2 * k], x = u[2 * k + 1];
            if (S.at[h].m < S.at[x].m) std::swap(h, x);
            S.cons.push_back({h, x, fl[k] * fl[k], 1.f / S.at[h].m + 1.f / S.at[x].m});
        }
    }
    std::fclose(f);
    S.w.resize(n);
    for (int i = 0; i < n; ++i) {
        Water& w = S.w[i];
        const float* p = &wp[9 * (size_t)i];
        const float* v = &wv[9 * (size_t)i];
        w.o = {p[0], p[1], p[2]}; w.h0 = {p[3], p[4], p[5]}; w.h1 = {p[6], p[7], p[8]};
        const V3 bis = (w.h0 - w.o) + (w.h1 - w.o);
        w.m = w.o + bis * (O_EP_R / std::sqrt(dot(bis, bis)));
        w.vo = {v[0], v[1], v[2]}; w.vh0 = {v[3], v[4], v[5]}; w.vh1 = {v[6], v[7], v[8]};
        w.ao = w.ah0 = w.ah1 = V3{0, 0, 0};
    }
    auto t0 = std::chrono::steady_clock::now();
    build_neighbors(S);
    all_forces(S);
    if (argc > 3) {
        // one force evaluation written out, for checking this restatement
        // against the float64 oracle: int32 n_water, n_atoms; float64 water
        // site forces [n][4][3] (O, H0, H1, M), atom forces [n_atoms][3];
        // float64 SPME energy (self term included), pair virial
        FILE* o = std::fopen(argv[3], "wb");
        if (!o) { std::fprintf(stderr, "cannot open %s\n", argv[3]); return 2; }
        const int32_t dims[2] = {n, na};
        std::fwrite(dims, 4, 2, o);
        for (const Water& w : S.w) {
            const V3 fs[4] = {w.fo, w.fh0, w.fh1, w.fm};
            for (const V3& v : fs) {
                const double d[3] = {v.x, v.y, v.z};
                std::fwrite(d, 8, 3, o);
            }
        }
        for (const Atom& a : S.at) {
            const double d[3] = {a.f.x, a.f.y, a.f.z};
            std::fwrite(d, 8, 3, o);
        }
        const double sc[2] = {S.spme_e, S.virial};
        std::fwrite(sc, 8, 2, o);
        std::fclose(o);
        return 0;
    }
    kick_calc_accel(S, 0.f);
    auto t_setup = std::chrono::steady_clock::now();
    const double budget = argc > 2 ? std::atof(argv[2]) : 1e30;
    for (int k = 0; k < warmup; ++k) step(S, dt);
    auto t1 = std::chrono::steady_clock::now();
    int done = 0;
    auto t2 = t1;
    for (; done < steps;) {
        step(S, dt);
        ++done;
        t2 = std::chrono::steady_clock::now();
        if (std::chrono::duration<double>(t2 - t1).count() > budget) break;
    }
    const int steps_run = done;
    const double sec = std::chrono::duration<double>(t2 - t1).count();
    const double setup = std::chrono::duration<double>(t_setup - t0).count();
    const double ns_day = steps_run * (double)dt * 1e-3 / sec * 86400.0;
    std::printf("{\"value\": %.6f, \"unit\": \"ns/day\", \"steps\": %d, \"warmup\": %d, \"seconds\": %.4f, "
                "\"setup_seconds\": %.4f, \"threads\": %d, \"pairs\": %zu, \"rebuilds\": %d, \"ke\": %.4f, "
                "\"pe_recip\": %.4f}\n",
                ns_day, steps_run, warmup, sec, setup, omp_get_max_threads(), S.pairs.size(), S.rebuilds, S.ke,
                S.spme_e);
    return 0;
}
