// xsmd.cpp -- process-level drop-in for the SMD part of the reference's
// xSMD_run, in C++ on the library's C ABI (libsmd_b200.so).
//
//   xsmd WORKDIR [--device D] [--precision fp64|fp32] [--stride S]
//        [--fix-every F] [--no-dwf-guard]
//
// Reads what the reference's main program reads from WORKDIR
// (Codes_Folder/smd_code.cpp:219-277, 472-539, 913-928, 997-1180): the five
// Settings_*.txt files, outBin/MC_Bin_SpinField<tag>.bin and, for the
// "wread" window, outBin/winvec.bin.  It integrates every sample on the GPU
// and writes the reference's output files with the same names, layouts and
// number formats:
//
//   outData/RK_Check/0WinTVec_<w>.dat, 0WinSpec_<w>.dat
//                     the temporal window and its ordered spectrum
//                     (smd_code.cpp:2808-2983)
//   outData/RK_Results/MCSamples_DFT_{xy,yz,zz,tt}Spec<tag>.dat and
//   outData/MC_Results/locFieldHist<tag>.dat
//                     the static pre-pass over the samples: centred static
//                     structure factor and local-field histograms
//                     (smd_code.cpp:2289-2726), on the GPU
//   outBin/MC_Bin_SpecData<tag>.bin
//                     sample-averaged spectra, per q the ntm doubles of x,
//                     y, z, then the autocorrelation (smd_code.cpp:3596-3631)
//   outData/MC_Results/SpinSpin_Temporal_Corr<tag>.dat
//                     time and autocorrelation (smd_code.cpp:4019-4033)
//   outData/RK_Results/DFT_{xy,yz,zz,tt}Spec_wfreq(<w>)<tag>.dat
//                     centred 2D spectra every ceil(npw / 10) bins
//                     (smd_code.cpp:3813-3855, subrouts.cpp:8868-9123)
//   outData/RK_Results/{KGMYG|YGMXG}_wDepn_DFT_{xy,yz,zz,tt}Spec<tag>.dat and
//                     {KGMCut|YGMCut}_wDepn_DFT_zzSpec<tag>.dat
//                     spectra along the high-symmetry path and its cut
//                     (smd_code.cpp:3700-3735, 3996-4130,
//                     subrouts.cpp:3688-3850, 9165-9280)
//
// with the quantum correction (smd_code.cpp:3645-3670) applied to the text
// spectra.  The reference assigns zVal twice there and never yVal, so its
// xy, yz and tt text outputs hold undefined values; this program applies the
// intended correction to x, y and z, and its zz outputs equal the
// reference's.  With RecVd1 = 2 in Settings_SMD_SIM.txt (the reference's
// getEvoData, subrouts.cpp:1840-1856) no evolution runs: the spectra come
// from an existing MC_Bin_SpecData file (smd_code.cpp:3532-3591) and only
// the text outputs are written.
//
// Defaults are the reference's semantics (FP64, every step recorded,
// correction every step); Settings_B200.txt ("fp32 4 16": precision,
// record stride, correction period) or the flags select the precision form.
#include "../../include/smd_b200.h"

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

const double kPi = std::acos(-1.0);
const double kPi2 = 2.0 * kPi;
const double kSq2 = std::sqrt(2.0);
const double kS60 = std::sin(kPi / 3.0);
const double kQval = 4.0 * kPi / 3.0;              // K point |Q|, subrouts.cpp:594
const double kBvec1[2] = {kPi2, -kPi / kS60};      // reciprocal vectors of the C3
const double kBvec2[2] = {0.0, kPi2 / kS60};       // lattices, subrouts.cpp:571-573
const char *kCodeSettings[16] = {"ptON",          "ptAdapt",      "ptTrack",       "ANNL_ON",
                                 "FFTW_ON",       "RKCheck",      "PBC_OFF",       "IsiModel",
                                 "qcrystal",      "with_recField", "with_DFTcodes", "force_Stripes",
                                 "refState_Zero", "qct_NeelPhase", "qct_RemovePBC", "rec_orderMaps"};
const int kBinSz = 1000;        // subrouts.cpp:309
const double kTempMax = 2.0;    // subrouts.cpp:389
const double kDwfMin = 0.10;    // subrouts.cpp:391

struct Fail : std::runtime_error {
    using std::runtime_error::runtime_error;
};

bool not_zero(double x) { return std::fabs(x) > 1.0e-12; }   // isNotZero, subrouts.cpp:773-778

std::vector<std::string> tokens(const std::string &path, size_t n)
{
    std::ifstream f(path);
    if (!f) throw Fail("cannot read " + path);
    std::vector<std::string> t;
    std::string s;
    while (t.size() < n && (f >> s)) t.push_back(s);
    if (t.size() < n) throw Fail(path + ": expected " + std::to_string(n) + " tokens");
    return t;
}

// The reference's settings files (subrouts.cpp:105-123, smd_code.cpp:497-539)
// and the derived quantities of convert_inputs2data that SMD uses.
struct Settings {
    int L = 0;
    double J1 = 1, J2 = 0, JX = 0, J2_delta = 0, zlamb1 = 1, zlamb2 = 1, h = 0, T1 = 0.1, T2 = 0.1;
    std::string geom;
    int NMeas = 0, crSkip = 1;
    std::string outTag;
    int ntm = 0, tpLstSz = 1, tpIndex = 0, RecVd1 = 0;
    double dtm = 0.01;
    std::string window;
    double imp_ratio = 0, J1ic = 0, J2ic = 0, JXic = 0, J1ii = 0, J2ii = 0, JXii = 0;
    int qcrystal = 0, pbc_off = 0, qct_rm_pbc = 0;

    int geom_id() const
    {
        static const char *g[5] = {"square", "triang", "hexagn", "kagome", "lieb"};
        for (int i = 0; i < 5; i++)
            if (geom == g[i]) return i;
        return -1;
    }
    // C3SYM, subrouts.cpp:1093-1096 (never for a quasi-crystal)
    bool c3() const { return !qcrystal && geom != "square" && geom != "lieb"; }
    bool disorder() const { return imp_ratio > 0.0; }
    bool j2_on() const
    {
        bool on = not_zero(J2) || not_zero(J2_delta);
        if (disorder()) on = on || not_zero(J2ic) || not_zero(J2ii);
        return on;
    }
    bool jx_on() const
    {
        bool on = not_zero(JX);
        if (disorder()) on = on || not_zero(JXic) || not_zero(JXii);
        return on;
    }
    int pack_size() const { return NMeas / crSkip; }   // smd_code.cpp:978
    double temperature() const
    {
        return tpLstSz > 1 ? T1 + tpIndex * (T2 - T1) / (tpLstSz - 1) : T1;
    }
    std::string tag() const   // "_T(%.5f)" + label, smd_code.cpp:913-928, subrouts.cpp:2158-2185
    {
        std::ostringstream o;
        o << std::fixed << std::setprecision(5) << temperature();
        std::ostringstream l;
        l << std::fixed << std::setprecision(3);
        if (outTag == "Htag") l << "_extH(" << h << ")";
        else if (outTag == "J1tag") l << "_J1(" << J1 << ")";
        else l << "_J2(" << J2 << ")";
        return "_T(" + o.str() + ")" + l.str();
    }

    void read(const std::string &dir)
    {
        auto c = tokens(dir + "/Settings_CodeExec.txt", 32);
        for (int i = 0; i < 16; i++) {
            const int v = std::stoi(c[2 * i + 1]);
            if (v != 0 && v != 1) throw Fail("invalid code-exec setting " + c[2 * i]);
            if (std::string(kCodeSettings[i]) == "qcrystal") qcrystal = v;
            if (std::string(kCodeSettings[i]) == "PBC_OFF") pbc_off = v;
            if (std::string(kCodeSettings[i]) == "qct_RemovePBC") qct_rm_pbc = v;
        }
        auto m = tokens(dir + "/Settings_MODEL.txt", 11);
        L = std::stoi(m[0]);
        J1 = std::stod(m[1]);
        J2 = std::stod(m[2]);
        JX = std::stod(m[3]);
        J2_delta = std::stod(m[4]);
        zlamb1 = std::stod(m[5]);
        zlamb2 = std::stod(m[6]);
        h = std::stod(m[7]);
        T1 = std::stod(m[8]);
        T2 = std::stod(m[9]);
        geom = m[10];
        auto s = tokens(dir + "/Settings_MC_SIM.txt", 8);
        NMeas = std::stoi(s[1]);
        outTag = s[4];
        crSkip = std::stoi(s[5]);
        auto d = tokens(dir + "/Settings_SMD_SIM.txt", 7);
        ntm = std::stoi(d[0]);
        tpLstSz = std::stoi(d[1]);
        tpIndex = std::stoi(d[2]);
        dtm = std::stod(d[3]);
        window = d[4];
        RecVd1 = std::stoi(d[5]);
        auto r = tokens(dir + "/Settings_Disorder.txt", 7);
        imp_ratio = std::stod(r[0]);
        J1ic = std::stod(r[1]);
        J2ic = std::stod(r[2]);
        JXic = std::stod(r[3]);
        J1ii = std::stod(r[4]);
        J2ii = std::stod(r[5]);
        JXii = std::stod(r[6]);
    }

    // the input checks of convert_inputs2data and main that apply to SMD
    void validate(bool check_dwf) const
    {
        if (qcrystal) {
            // latSize is the site count of an approximant (subrouts.cpp:
            // 1005-1114); the run needs PBC_OFF = 1 and qct_RemovePBC = 0
            // (smd_code.cpp:365-372)
            if (geom != "Aamman") throw Fail("unknown quasi-geometry " + geom);
            if (qct_rm_pbc || !pbc_off) throw Fail("qcrystal needs PBC_OFF = 1 and qct_RemovePBC = 0");
            if (L < 4) throw Fail("quasi-crystal size too small");
        } else {
            if (geom_id() < 0) throw Fail("unknown geometry " + geom);
            if (L % 2) throw Fail("lattice length must be a multiple of 2");
            if (c3() && L % 3) throw Fail("lattice length must be a multiple of 3");
        }
        if (not_zero(J2_delta) && geom != "lieb") throw Fail("J2_delta requires the lieb geometry");
        if (NMeas % kBinSz || NMeas / kBinSz == 1) throw Fail("NMeas must be a multiple of BinSz with more than one bin");
        if (crSkip <= 0 || kBinSz % crSkip || crSkip > kBinSz) throw Fail("crSkip must divide BinSz");
        if (ntm < 10) throw Fail("ntm too small");
        if (dtm > 0.05) throw Fail("dtm too large");
        static const char *w[11] = {"wread", "gauss", "ntall", "black", "flatw", "hann1",
                                    "sincw", "hann2", "lancz", "hann3", "nowin"};
        if (std::find_if(w, w + 11, [&](const char *x) { return window == x; }) == w + 11)
            throw Fail("invalid window " + window);
        if (!(imp_ratio >= 0.0 && imp_ratio < 1.0)) throw Fail("impurity ratio must lie in [0, 1)");
        if (tpIndex < 0 || tpIndex >= tpLstSz) throw Fail("tpIndex outside the temperature list");
        if (temperature() > kTempMax) throw Fail("temperature exceeds TempMax");
        const double dwf = 2.0 * kPi / (ntm * dtm);
        if (check_dwf && dwf > kDwfMin) throw Fail("dwf exceeds dwf_min (use --no-dwf-guard)");
    }
};

void mkdirs(const std::string &p)
{
    std::string cur;
    std::stringstream ss(p);
    std::string part;
    while (std::getline(ss, part, '/')) {
        if (part.empty()) {
            cur += "/";
            continue;
        }
        cur += part + "/";
        if (::mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) throw Fail("cannot create " + cur);
    }
}

// C++ `scientific << showpos << setprecision(dg) << setw(wd)` (fmtDbleSci,
// aux_code.cpp:545-556)
std::string sci(double x, int dg, int wd)
{
    std::ostringstream o;
    o << std::scientific << std::showpos << std::setprecision(dg) << std::setw(wd) << x;
    return o.str();
}

// The reference's sample file: per pack an int32 impurity map (disorder)
// then PackSize spin fields of N x 3 doubles (smd_code.cpp:997-1066).
void read_samples(const std::string &path, const Settings &s, int N, std::vector<double> &spins,
                  std::vector<int> &imp, int &n)
{
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw Fail("cannot read " + path);
    const size_t size = (size_t)f.tellg();
    f.seekg(0);
    const size_t conf = (size_t)N * 3 * 8, P = (size_t)s.pack_size();
    const size_t pack = (s.disorder() ? (size_t)N * 4 : 0) + P * conf;
    const size_t ref = s.disorder() ? pack : conf;
    size_t n_packs;
    if (size == ref) n_packs = 1;
    else if (size % ref) throw Fail(path + ": size is not a multiple of the configuration size");
    else {
        n_packs = size / pack;
        if (n_packs * P != (size - (s.disorder() ? n_packs * N * 4 : 0)) / conf)
            throw Fail(path + ": inconsistent pack layout");
    }
    const size_t first = (size == conf && !s.disorder()) ? 1 : P;
    n = 0;
    std::vector<int> map((size_t)N);
    for (size_t p = 0; p < n_packs; p++) {
        if (s.disorder()) f.read(reinterpret_cast<char *>(map.data()), (std::streamsize)N * 4);
        const size_t cnt = p == 0 ? first : P;
        const size_t off = spins.size();
        spins.resize(off + cnt * N * 3);
        f.read(reinterpret_cast<char *>(spins.data() + off), (std::streamsize)(cnt * conf));
        if (s.disorder())
            for (size_t k = 0; k < cnt; k++) imp.insert(imp.end(), map.begin(), map.end());
        n += (int)cnt;
    }
    if (!f) throw Fail(path + ": short read");
}

void check(int rc, smd_ctx *ctx, const char *what)
{
    if (rc != SMD_OK)
        throw Fail(std::string(what) + " failed (" + std::to_string(rc) + ")" +
                   (ctx ? std::string(": ") + smd_last_error(ctx) : std::string()));
}

// FFT-order index -> centred order (get_OrderedSpecArray1D / 2D,
// subrouts.cpp:8868-8962): index i of the ordered array reads i + n/2 for
// i < n/2, i - n/2 otherwise
int centred(int i, int n)
{
    const int l2 = n / 2;
    const int m = 2 * (i / l2);
    return i - l2 * (m - 1);
}

// radix-2 / direct DFT of the window (forward, unnormalised); lengths that
// are not powers of two use the direct sum
std::vector<std::complex<double>> dft(const std::vector<double> &x)
{
    const size_t n = x.size();
    std::vector<std::complex<double>> a(x.begin(), x.end());
    if (n && !(n & (n - 1))) {
        for (size_t i = 1, j = 0; i < n; i++) {
            size_t bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) std::swap(a[i], a[j]);
        }
        for (size_t len = 2; len <= n; len <<= 1) {
            for (size_t i = 0; i < n; i += len)
                for (size_t k = 0; k < len / 2; k++) {
                    const double ang = -kPi2 * (double)k / (double)len;
                    const std::complex<double> w(std::cos(ang), std::sin(ang));
                    const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                    a[i + k] = u + v;
                    a[i + k + len / 2] = u - v;
                }
        }
        return a;
    }
    std::vector<std::complex<double>> out(n);
    for (size_t k = 0; k < n; k++) {
        std::complex<double> s = 0.0;
        for (size_t t = 0; t < n; t++) {
            const double ang = -kPi2 * (double)((k * t) % n) / (double)n;
            s += x[t] * std::complex<double>(std::cos(ang), std::sin(ang));
        }
        out[k] = s;
    }
    return out;
}

// The window of the run (smd_code.cpp:2818-2880; "wread" rescales the file's
// values by their maximum) and its two record files (smd_code.cpp:2940-2983).
std::vector<double> window_and_files(const Settings &s, const std::string &dir, int n)
{
    std::vector<double> w((size_t)n);
    if (s.window == "wread") {
        std::ifstream f(dir + "/outBin/winvec.bin", std::ios::binary);
        if (!f) throw Fail("cannot read outBin/winvec.bin");
        f.read(reinterpret_cast<char *>(w.data()), (std::streamsize)n * 8);
        if (!f) throw Fail("outBin/winvec.bin holds fewer than ntm values");
        double mx = 0.0;
        for (double v : w) mx = v > mx ? v : mx;
        const double fc = 1.0 / mx;
        for (double &v : w) v = fc * v;
    } else {
        check(smd_window(s.window.c_str(), n, w.data()), nullptr, "smd_window");
    }
    mkdirs(dir + "/outData/RK_Check");
    const auto X = dft(w);
    std::vector<double> p0((size_t)n), p1((size_t)n);
    for (int k = 0; k < n; k++) p0[k] = (1.0 / n) * std::norm(X[k]);
    for (int k = 0; k < n; k++) p1[k] = p0[centred(k, n)];
    double ref = p1[0];
    for (int k = 1; k < n; k++) ref = p1[k] > ref ? p1[k] : ref;
    std::ofstream f1(dir + "/outData/RK_Check/0WinTVec_" + s.window + ".dat");
    std::ofstream f2(dir + "/outData/RK_Check/0WinSpec_" + s.window + ".dat");
    const double fs0 = 2.0 / n;
    for (int k = 0; k < n; k++) {
        f1 << k * s.dtm << "   " << w[k] << "\n";
        f2 << k * fs0 - 1.0 << "   " << std::log10(p1[k] / ref) << "\n";
    }
    return w;
}

// ------------------------------------------------------------- outputs

struct Grid {
    int G = 0;
    bool c3 = false;
    double dq = 0.0;   // pi2 / Gsz, smd_code.cpp:1774
};

// centred component arrays of one frequency bin (get_OrderedSpecArray2D,
// subrouts.cpp:8868-8927): xy = (x + y) / 2, yz = (y + z) / 2,
// tt = (x + y + z) / 3, zz = z
void ordered(const Grid &g, const double *x, const double *y, const double *z, size_t ntm, int n,
             std::vector<double> a[4])
{
    const int G = g.G;
    for (int k = 0; k < 4; k++) a[k].assign((size_t)G * G, 0.0);
    for (int i = 0; i < G; i++) {
        const int m1 = centred(i, G);
        for (int j = 0; j < G; j++) {
            const size_t q = (size_t)m1 * G + centred(j, G);
            const double vx = x[q * ntm + n], vy = y[q * ntm + n], vz = z[q * ntm + n];
            const size_t o = (size_t)i * G + j;
            a[0][o] = (1.0 / 2.0) * (vx + vy);
            a[1][o] = (1.0 / 2.0) * (vy + vz);
            a[2][o] = vz;
            a[3][o] = (1.0 / 3.0) * (vx + vy + vz);
        }
    }
}

// the path's grid points in the centred arrays (get_Spec_qPath,
// subrouts.cpp:9165-9280)
std::vector<std::pair<int, int>> path_points(const Grid &g)
{
    const int G = g.G, l2 = G / 2;
    std::vector<std::pair<int, int>> p;
    if (g.c3) {
        for (int j = l2 / 3; j <= l2; j++) p.push_back({G - j, j});     // K -> G
        for (int j = l2 - 1; j >= 0; j--) p.push_back({l2, j});        // G -> M
        for (int j = 1; j <= l2 / 2; j++) p.push_back({l2 - j, j});    // M -> Y
        for (int i = l2 / 2 + 1; i <= l2; i++) p.push_back({i, i});    // Y -> G
    } else {
        for (int j = 0; j <= l2; j++) p.push_back({l2, j});            // Y -> G
        for (int i = l2 - 1; i >= 0; i--) p.push_back({i, i});         // G -> M
        for (int j = 1; j <= l2; j++) p.push_back({0, j});             // M -> X
        for (int i = 1; i <= l2; i++) p.push_back({i, l2});            // X -> G
    }
    return p;
}

// the path's wavevectors (get_qPathWVectors, subrouts.cpp:3688-3850) and
// their cumulative length along the path (smd_code.cpp:3996-4015)
std::vector<double> path_lengths(const Grid &g)
{
    const int G = g.G, l2 = G / 2;
    const double fc = 1.0 / G;
    const double b1[2] = {fc * kBvec1[0], fc * kBvec1[1]}, b2[2] = {fc * kBvec2[0], fc * kBvec2[1]};
    std::vector<std::pair<double, double>> w;
    auto grid_q = [&](int i, int j) {
        const int m1 = i - l2, m2 = j - l2;
        w.push_back({m1 * b1[0] + m2 * b2[0], m1 * b1[1] + m2 * b2[1]});
    };
    if (g.c3) {
        for (int j = l2 / 3; j <= l2; j++) grid_q(G - j, j);
        for (int j = l2 - 1; j >= 0; j--) grid_q(l2, j);
        for (int j = 1; j <= l2 / 2; j++) grid_q(l2 - j, j);
        for (int i = l2 / 2 + 1; i <= l2; i++) grid_q(i, i);
    } else {
        const double dq = g.dq;
        for (int i = 0; i < l2; i++) w.push_back({0.0, i * dq - kPi});   // Y -> G
        std::vector<std::pair<double, double>> v;                       // G -> X -> M -> G, reversed
        for (int j = l2; j >= 0; j--) v.push_back({j * dq - kPi, 0.0});
        for (int i = l2 - 1; i >= 0; i--) v.push_back({-kPi, i * dq - kPi});
        for (int i = 1; i <= l2; i++) v.push_back({i * dq - kPi, i * dq - kPi});
        std::reverse(v.begin(), v.end());
        w.insert(w.end(), v.begin(), v.end());
    }
    std::vector<double> len(w.size());
    double ref0 = w[0].first, ref1 = w[0].second, acc = 0.0;
    for (size_t k = 0; k < w.size(); k++) {
        const double qx = w[k].first - ref0, qy = w[k].second - ref1;
        acc = acc + std::sqrt(std::pow(qx, 2) + std::pow(qy, 2));
        len[k] = acc;
        ref0 = w[k].first;
        ref1 = w[k].second;
    }
    return len;
}

// hexagonal first-zone filter (hexFilter, aux_code.cpp:1189-1215)
bool hex_filter(double qx, double qy, double Q0, double dQ)
{
    const double sq3 = std::sqrt(3.0), s60 = 0.5 * sq3;
    const double Qs = Q0 + dQ / 3.0;
    if (std::fabs(qy) - Qs * s60 < 0.0) {
        const double w1 = sq3 * (qx - Qs) - qy, w2 = sq3 * (qx - Qs) + qy;
        const double w3 = sq3 * (qx + Qs) - qy, w4 = sq3 * (qx + Qs) + qy;
        return (w1 < 0.0 && w2 < 0.0) && (w3 > 0.0 && w4 > 0.0);
    }
    return false;
}

// one centred 2D spectrum as text (record_SpecArray2D, subrouts.cpp:8979-9123)
void record_2d(const Grid &g, const std::vector<double> &a, const std::string &path)
{
    std::ofstream f(path);
    const int sz = g.G, l2 = sz / 2;
    const double fc = 1.0 / sz;
    const double b1[2] = {fc * kBvec1[0], fc * kBvec1[1]}, b2[2] = {fc * kBvec2[0], fc * kBvec2[1]};
    if (g.c3) {
        const double q1[2] = {l2 * b1[0], l2 * b1[1]}, q2[2] = {l2 * b2[0], l2 * b2[1]};
        for (int n1 = 0; n1 < 3; n1++) {
            const int m1s = 2 * (n1 - 1);
            for (int i = 0; i < sz; i++) {
                for (int n2 = 0; n2 < 3; n2++) {
                    const int m2s = 2 * (n2 - 1);
                    const double qx0 = m1s * q1[0] + m2s * q2[0], qy0 = m1s * q1[1] + m2s * q2[1];
                    for (int j = 0; j < sz; j++) {
                        const double pw = a[(size_t)i * sz + j];
                        const int m1 = i - l2, m2 = j - l2;
                        const double qx = qx0 + (m1 * b1[0] + m2 * b2[0]);
                        const double qy = qy0 + (m1 * b1[1] + m2 * b2[1]);
                        if (hex_filter(qx, qy, kQval, g.dq)) f << qx << "   " << qy << "   " << pw << "\n";
                        else f << qx << "   " << qy << "   " << "NaN" << "\n";
                    }
                }
                f << "\n";
            }
        }
    } else {
        for (int i = 0; i <= sz; i++) {
            for (int j = 0; j <= sz; j++) {
                const double pw = a[(size_t)(i % sz) * sz + (j % sz)];
                f << g.dq * (i - l2) << "   " << g.dq * (j - l2) << "   " << pw << "\n";
            }
            f << "\n";
        }
    }
}

// C++ `fixed << showpos << setprecision(dg) << setw(wd)` (fmtDbleFix,
// aux_code.cpp:530-541)
std::string fix(double x, int dg, int wd)
{
    std::ostringstream o;
    o << std::fixed << std::showpos << std::setprecision(dg) << std::setw(wd) << x;
    return o.str();
}

// The static pre-pass records (smd_code.cpp:2641-2696): the centred static
// structure factor MCSamples_DFT_{xy,yz,zz,tt}Spec and the local-field
// histograms locFieldHist.  sf [3][G*G], hist [201][3] counts.
void write_prepass(const Settings &s, const std::string &dir, const std::string &tag, int G,
                   const std::vector<double> &sf, const std::vector<long long> &hist, double r0)
{
    const std::string res = dir + "/outData/RK_Results/", mcr = dir + "/outData/MC_Results/";
    mkdirs(res);
    mkdirs(mcr);
    Grid g;
    g.G = G;
    g.c3 = s.c3();
    g.dq = kPi2 / G;
    const size_t Q = (size_t)G * G;
    std::vector<double> a[4];
    ordered(g, sf.data(), sf.data() + Q, sf.data() + 2 * Q, 1, 0, a);
    const char *comp[4] = {"xy", "yz", "zz", "tt"};
    for (int c = 0; c < 4; c++) record_2d(g, a[c], res + "MCSamples_DFT_" + comp[c] + "Spec" + tag + ".dat");
    const int nh = 201;
    const double box = 2.0 * r0 / (nh - 1);
    double norm[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < nh; k++)
        for (int c = 0; c < 3; c++) norm[c] += (double)hist[(size_t)k * 3 + c];
    std::ofstream f(mcr + "locFieldHist" + tag + ".dat");
    for (int k = 0; k < nh; k++) {
        f << fix(k * box - r0, 4, 8) << "  ";
        for (int c = 0; c < 3; c++) f << fix((double)hist[(size_t)k * 3 + c] / norm[c], 4, 10) << "  ";
        f << "\n";
    }
}

// The text outputs of smd_code.cpp:3640-4130 from the sample-averaged
// spectra spec [3][Q][ntm] and autocorrelation qss [ntm].
void write_text(const Settings &s, const std::string &dir, const std::string &tag, int G, int ntm, double dtm_rec,
                std::vector<double> spec, const std::vector<double> &qss)
{
    const std::string res = dir + "/outData/RK_Results/", mcr = dir + "/outData/MC_Results/";
    mkdirs(res);
    mkdirs(mcr);
    Grid g;
    g.G = G;
    g.c3 = s.c3();
    g.dq = kPi2 / G;
    const size_t Q = (size_t)G * G;
    // quantum correction: itFac * qtFac(beta w) for every component
    const double tmax = ntm * dtm_rec, dwf = 2.0 * kPi / tmax, itFac = tmax / kPi2;
    const double beta = 1.0 / s.temperature();
    for (size_t k = 0; k < Q; k++)
        for (int n = 0; n < ntm; n++) {
            const double fc = beta * (n * dwf);
            const double qt = n > 0 ? fc / (1.0 - std::exp(-fc)) : 1.0;
            for (int c = 0; c < 3; c++) {
                double &v = spec[(c * Q + k) * ntm + n];
                v = itFac * qt * v;
            }
        }
    const double *x = spec.data(), *y = x + Q * ntm, *z = y + Q * ntm;
    const int npw = ntm / 2, nmax = npw;
    const auto pts = path_points(g);
    const size_t np = pts.size();
    std::vector<double> path[4];
    for (auto &p : path) p.assign(np * npw, 0.0);
    std::vector<double> a[4];
    const char *comp[4] = {"xy", "yz", "zz", "tt"};
    const int skip = (int)std::ceil(0.1 * nmax);
    for (int n = 0; n < npw; n++) {
        ordered(g, x, y, z, ntm, n, a);
        for (int c = 0; c < 4; c++)
            for (size_t j = 0; j < np; j++) path[c][j * npw + n] = a[c][(size_t)pts[j].first * G + pts[j].second];
        if (n % skip == 0) {
            std::ostringstream w;
            w << std::fixed << std::setprecision(3) << n * dwf;
            for (int c = 0; c < 4; c++)
                record_2d(g, a[c], res + "DFT_" + comp[c] + "Spec_wfreq(" + w.str() + ")" + tag + ".dat");
        }
    }
    // autocorrelation
    {
        std::ofstream f(mcr + "SpinSpin_Temporal_Corr" + tag + ".dat");
        for (int n = 0; n < ntm; n++) f << sci(n * dtm_rec, 8, 15) << "    " << sci(qss[n], 12, 22) << "\n";
    }
    // path and cut files
    const auto len = path_lengths(g);
    const std::string pre = g.c3 ? "KGMYG" : "YGMXG", cut = g.c3 ? "KGMCut" : "YGMCut";
    const double cut1 = g.c3 ? 0.0 : kPi * 0.5, cut2 = g.c3 ? kPi : kPi * (1.0 + 0.5 * kSq2);
    std::ofstream f[4], fc5(res + cut + "_wDepn_DFT_zzSpec" + tag + ".dat");
    for (int c = 0; c < 4; c++) f[c].open(res + pre + "_wDepn_DFT_" + comp[c] + "Spec" + tag + ".dat");
    for (size_t k = 0; k < np; k++) {
        const double lp = len[k];
        for (int n = 0; n < nmax; n++) {
            const double wf = n * dwf;
            for (int c = 0; c < 4; c++)
                f[c] << sci(lp, 8, 15) << "    " << sci(wf, 8, 15) << "    " << sci(path[c][k * npw + n], 12, 22)
                     << "\n";
            if (lp >= cut1 && lp <= cut2)
                fc5 << sci(lp, 8, 15) << "    " << sci(wf, 8, 15) << "    " << sci(path[2][k * npw + n], 12, 22)
                    << "\n";
        }
        for (int c = 0; c < 4; c++) f[c] << "\n";
        fc5 << "\n";
    }
}

// The autocorrelation file alone (smd_code.cpp:4019-4033): the text spectra
// of the output stage assume a Bravais grid and are written for crystals only.
void write_corr(const std::string &dir, const std::string &tag, int ntm, double dtm_rec,
                const std::vector<double> &qss)
{
    const std::string mcr = dir + "/outData/MC_Results/";
    mkdirs(mcr);
    std::ofstream f(mcr + "SpinSpin_Temporal_Corr" + tag + ".dat");
    for (int n = 0; n < ntm; n++) f << sci(n * dtm_rec, 8, 15) << "    " << sci(qss[n], 12, 22) << "\n";
}

// A quasi-crystal's tables from outBin/ (smd_code.cpp:1248-1300 and
// 1575-1660): sitesList (N x 2 doubles) and nborsList (per site Zn1, Zn2,
// ZnX int32, -1 ghosts), exact sizes, unit nearest-neighbour spacing
// (check_latticeSpc, subrouts.cpp:5803-5832: entries > 0 of site 0).
void read_qct_tables(const std::string &dir, int N, const int zn[3], std::vector<double> &rvec,
                     std::vector<int> nb[3])
{
    const std::string tag = "_AppxtSz(" + std::to_string(N) + ")";
    const std::string sites = dir + "/outBin/sitesList" + tag + ".bin", nbors = dir + "/outBin/nborsList" + tag + ".bin";
    std::ifstream fs(sites, std::ios::binary | std::ios::ate), fn(nbors, std::ios::binary | std::ios::ate);
    const int zt = zn[0] + zn[1] + zn[2];
    if (!fs || (size_t)fs.tellg() != (size_t)N * 16) throw Fail("invalid or missing " + sites);
    if (!fn || (size_t)fn.tellg() != (size_t)N * zt * 4) throw Fail("invalid or missing " + nbors);
    fs.seekg(0);
    fn.seekg(0);
    fs.read(reinterpret_cast<char *>(rvec.data()), (std::streamsize)N * 16);
    std::vector<int> row((size_t)zt);
    for (int i = 0; i < N; i++) {
        fn.read(reinterpret_cast<char *>(row.data()), (std::streamsize)zt * 4);
        int o = 0;
        for (int k = 0; k < 3; k++)
            for (int q = 0; q < zn[k]; q++, o++) {
                if (row[o] >= N) throw Fail(nbors + ": neighbour index out of range");
                nb[k][(size_t)i * zn[k] + q] = row[o];
            }
    }
    double lspc = 100.0;
    for (int q = 0; q < zn[0]; q++) {
        const int j = nb[0][q];
        if (j > 0) lspc = std::min(lspc, std::hypot(rvec[2 * j] - rvec[0], rvec[2 * j + 1] - rvec[1]));
    }
    if (lspc < 0.95 || lspc > 1.05) throw Fail("lattice spacing is not unit");
}

int usage()
{
    std::cerr << "usage: xsmd WORKDIR [--device D] [--precision fp64|fp32] [--stride S] [--fix-every F]"
                 " [--no-dwf-guard]\n";
    return 2;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) return usage();
    const std::string dir = argv[1];
    int device = 0, stride = 1, fix_every = 1, prec = SMD_FP64;
    bool dwf_guard = true, have_p = false, have_s = false, have_f = false;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) throw Fail("missing value after " + a);
            return argv[++i];
        };
        try {
            if (a == "--device") device = std::stoi(next());
            else if (a == "--precision") {
                const std::string v = next();
                if (v != "fp64" && v != "fp32") return usage();
                prec = v == "fp32" ? SMD_FP32 : SMD_FP64;
                have_p = true;
            } else if (a == "--stride") stride = std::stoi(next()), have_s = true;
            else if (a == "--fix-every") fix_every = std::stoi(next()), have_f = true;
            else if (a == "--no-dwf-guard") dwf_guard = false;
            else return usage();
        } catch (const std::exception &e) {
            std::cerr << "xsmd: " << e.what() << "\n";
            return 2;
        }
    }
    smd_ctx *ctx = nullptr;
    try {
        Settings s;
        s.read(dir);
        s.validate(dwf_guard);
        {
            // optional precision-form settings: "fp32 4 16"
            std::ifstream o(dir + "/Settings_B200.txt");
            std::string p;
            int st = 0, fe = 0;
            if (o >> p >> st >> fe) {
                if (!have_p) prec = p == "fp32" ? SMD_FP32 : SMD_FP64;
                if (!have_s) stride = st;
                if (!have_f) fix_every = fe;
            }
        }
        if (stride < 1 || fix_every < 1) throw Fail("stride and correction period must be positive");
        const std::string tag = s.tag();
        int N = 0, G = 0, nsubs = 0, zn[3] = {0, 0, 0};
        if (s.qcrystal) {
            // Ammann-Beenker tables: Zn = (8, 3, 8) (subrouts.cpp:1006-1012);
            // the direct-sum q set is Lsz x Lsz, Lsz the even integer below
            // sqrt(N) (subrouts.cpp:1111)
            N = s.L;
            zn[0] = 8;
            zn[1] = 3;
            zn[2] = 8;
            nsubs = 1;
            G = ((int)std::sqrt((double)N) / 2) * 2;
        } else {
            check(smd_geometry_info(s.geom_id(), s.L, &N, &G, &nsubs, zn), nullptr, "smd_geometry_info");
        }
        const int n_rec = stride == 1 ? s.ntm : (s.ntm - 1) / stride + 1;
        const int Q = G * G;
        std::vector<double> spec((size_t)3 * Q * n_rec), qss((size_t)n_rec);
        const std::string bin = dir + "/outBin/MC_Bin_SpecData" + tag + ".bin";
        std::vector<double> win = window_and_files(s, dir, s.ntm);
        auto t0 = std::chrono::steady_clock::now();
        double drift = 0.0;
        int n = 0;
        if (s.RecVd1 == 2) {
            // getEvoData: the spectra of an earlier run, smd_code.cpp:3532-3591
            std::ifstream f(bin, std::ios::binary | std::ios::ate);
            if (!f) throw Fail("could not find input file " + bin);
            const size_t want = (size_t)(3 * Q + 1) * s.ntm * 8;
            if ((size_t)f.tellg() != want) throw Fail(bin + ": input file has no valid data");
            f.seekg(0);
            std::vector<double> row((size_t)s.ntm);
            for (int k = 0; k < Q; k++)
                for (int c = 0; c < 3; c++) {
                    f.read(reinterpret_cast<char *>(row.data()), (std::streamsize)s.ntm * 8);
                    std::copy(row.begin(), row.end(), spec.begin() + ((size_t)c * Q + k) * s.ntm);
                }
            f.read(reinterpret_cast<char *>(qss.data()), (std::streamsize)s.ntm * 8);
        } else {
            std::vector<double> rvec((size_t)N * 2);
            std::vector<int> gmap((size_t)Q), nb[3];
            for (int k = 0; k < 3; k++) nb[k].assign((size_t)N * zn[k], -1);
            if (s.qcrystal) read_qct_tables(dir, N, zn, rvec, nb);
            else
                check(smd_build_lattice(s.geom_id(), s.L, rvec.data(), gmap.data(), nb[0].data(), nb[1].data(),
                                        nb[2].data()),
                      nullptr, "smd_build_lattice");
            const int maxb = N * (zn[0] + zn[1] + zn[2]);
            std::vector<int> bonds((size_t)maxb * 2);
            int nbonds[4];
            check(smd_build_bonds(N, zn, nb[0].data(), nb[1].data(), nb[2].data(), s.j2_on(), s.jx_on(),
                                  bonds.data(), maxb, nbonds),
                  nullptr, "smd_build_bonds");
            std::vector<double> spins;
            std::vector<int> imp;
            read_samples(dir + "/outBin/MC_Bin_SpinField" + tag + ".bin", s, N, spins, imp, n);
            smd_device_opts o{device, 0};
            check(smd_ctx_create(&o, &ctx), nullptr, "smd_ctx_create (needs a B200)");
            smd_lattice_desc d{};
            d.N = N;
            for (int k = 0; k < 3; k++) {
                d.zn[k] = zn[k];
                d.nbr[k] = nb[k].data();
            }
            d.shell_on[0] = 1;
            d.shell_on[1] = s.j2_on();
            d.shell_on[2] = s.jx_on();
            // couplings J[shell][a_i][a_j] (subrouts.cpp:2093-2099) and lambda
            // vectors (subrouts.cpp:2112-2133)
            const double cc[3] = {s.J1, s.J2, s.JX};
            const double ic[3] = {s.J1ic, s.J2ic, s.JXic}, ii[3] = {s.J1ii, s.J2ii, s.JXii};
            for (int k = 0; k < 3; k++) {
                d.J[k][0][0] = cc[k];
                d.J[k][0][1] = d.J[k][1][0] = s.disorder() ? ic[k] : 0.0;
                d.J[k][1][1] = s.disorder() ? ii[k] : 0.0;
                const bool xxz = s.zlamb1 != 1.0 || s.zlamb2 != 1.0;
                d.lambda[k][0] = d.lambda[k][1] = 1.0;
                d.lambda[k][2] = xxz ? (k == 0 ? s.zlamb1 : s.zlamb2) : 1.0;
            }
            d.lieb_delta_on = not_zero(s.J2_delta);
            d.j2_delta = s.J2_delta;
            d.h = s.h;
            for (int k = 0; k < 3; k++) d.nbonds[k] = nbonds[k + 1];
            d.bonds = bonds.data();
            d.G = s.qcrystal ? 0 : G;
            d.grid_map = s.qcrystal ? nullptr : gmap.data();
            d.pos = rvec.data();
            int lid = 0, qid = 0;
            check(smd_lattice_upload(ctx, &d, &lid), ctx, "smd_lattice_upload");
            if (s.qcrystal) {
                // get_qct_SqData (subrouts.cpp:8460-8525): index j Lsz + i
                // holds q = dq (nx(i), ny(j)), n in FFT order, dq = 4 pi2 / Lsz
                // (smd_code.cpp:1774), scale 1 / sqrt(N)
                std::vector<double> ql((size_t)Q * 2);
                const double dq = 4.0 * kPi2 / G;
                for (int jy = 0; jy < G; jy++)
                    for (int ix = 0; ix < G; ix++) {
                        const int nx = ix < G / 2 ? ix : ix - G, ny = jy < G / 2 ? jy : jy - G;
                        ql[((size_t)jy * G + ix) * 2] = nx * dq;
                        ql[((size_t)jy * G + ix) * 2 + 1] = ny * dq;
                    }
                check(smd_qset_upload(ctx, lid, 0, Q, ql.data(), 1.0 / std::sqrt((double)N), &qid), ctx,
                      "smd_qset_upload");
            } else {
                check(smd_qset_upload(ctx, lid, 1, 0, nullptr, 1.0, &qid), ctx, "smd_qset_upload");
            }
            // the static pre-pass over every sample (smd_code.cpp:2289-2726);
            // a quasi-crystal's runs over the direct-sum q set, not built here
            if (!s.qcrystal) {
                std::vector<double> sf((size_t)3 * Q);
                std::vector<long long> hist(201 * 3);
                double r0 = 0.0;
                check(smd_static_prepass(ctx, lid, qid, n, spins.data(), imp.empty() ? nullptr : imp.data(),
                                         sf.data(), hist.data(), &r0),
                      ctx, "smd_static_prepass");
                write_prepass(s, dir, tag, G, sf, hist, r0);
            }
            smd_job_desc j{};
            j.lattice = lid;
            j.qset = qid;
            j.n_samples = n;
            j.dt = s.dtm;
            j.n_rec = n_rec;
            j.stride = stride;
            j.precision = prec;
            j.fix_every = fix_every;
            j.imp = imp.empty() ? nullptr : imp.data();
            smd_report rep{};
            check(smd_run(ctx, &j, spins.data(), win.data(), spec.data(), qss.data(), nullptr, &rep), ctx,
                  "smd_run");
            drift = rep.drift_max;
            smd_ctx_destroy(ctx);
            ctx = nullptr;
            // the averaged spectra in the reference's checkpoint layout
            mkdirs(dir + "/outBin");
            std::remove(bin.c_str());
            std::ofstream f(bin, std::ios::binary);
            for (int k = 0; k < Q; k++)
                for (int c = 0; c < 3; c++)
                    f.write(reinterpret_cast<const char *>(spec.data() + ((size_t)c * Q + k) * n_rec),
                            (std::streamsize)n_rec * 8);
            f.write(reinterpret_cast<const char *>(qss.data()), (std::streamsize)n_rec * 8);
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (s.qcrystal) write_corr(dir, tag, n_rec, s.dtm * stride, qss);
        else write_text(s, dir, tag, G, n_rec, s.dtm * stride, spec, qss);
        std::cout << "{\"samples\": " << n << ", \"N\": " << N << ", \"Q\": " << Q << ", \"records\": " << n_rec
                  << ", \"precision\": \"" << (prec == SMD_FP32 ? "fp32" : "fp64") << "\", \"stride\": " << stride
                  << ", \"fix_every\": " << fix_every << ", \"resumed\": " << (s.RecVd1 == 2 ? "true" : "false")
                  << ", \"wall_s\": " << wall << ", \"drift_max_per_site\": " << drift << "}\n";
        return 0;
    } catch (const std::exception &e) {
        if (ctx) smd_ctx_destroy(ctx);
        std::cerr << "xsmd: " << e.what() << "\n";
        return 1;
    }
}
