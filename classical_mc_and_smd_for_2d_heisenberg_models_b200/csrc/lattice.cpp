// lattice.cpp -- host-side lattice tables, bond list and temporal windows.
//
// The tables are the input contract of the SMD path: neighbour order fixes
// the summation order of the local field and the d-wave sign of the Lieb J2
// term (Codes_Folder/subrouts.cpp:4527-4531), and nborsList.bin is written in
// this order.  So the tables must equal the reference's entry for entry.
// The reference finds neighbours by an O(N^2) scan of all sites and their
// eight periodic images (Codes_Folder/subrouts.cpp:2983-3316); here each
// site only scans the sites of the surrounding cells.  Every quantity that
// decides membership, order or rotation is computed from the same integer
// coordinates and with the same floating-point operations as the reference,
// so the result is identical:
//   - coordinates: round(500 * r) (subrouts.cpp:3036-3044)
//   - image shifts: subrouts.cpp:3066-3112
//   - shells by floor(distance) against floor(500 * 1.10), floor(500 * f2 *
//     1.05), floor(1000 * 1.05) (subrouts.cpp:3138-3200)
//   - order: angle atan2(dy, dx) descending (subrouts.cpp:3226-3228)
//   - hexagn / kagome rotations (subrouts.cpp:3230-3270), where the kagome
//     average angle is summed in the reference's scan order.
#include "../../include/smd_b200.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

namespace {

const double kPi = std::acos(-1.0);

struct Geo {
    int nsubs, grid_fac, zn[3];
};

bool geometry(int geom, Geo &g)
{
    switch (geom) {
    case SMD_SQUARE: g = {1, 1, {4, 4, 4}}; return true;
    case SMD_TRIANG: g = {1, 1, {6, 6, 6}}; return true;
    case SMD_HEXAGN: g = {2, 3, {3, 6, 3}}; return true;
    case SMD_KAGOME: g = {3, 2, {4, 4, 6}}; return true;
    case SMD_LIEB: g = {2, 2, {4, 4, 4}}; return true;
    default: return false;
    }
}

double size_factor(int geom)
{
    switch (geom) {
    case SMD_HEXAGN: return std::sqrt(3.0);
    case SMD_KAGOME: return 2.0;
    case SMD_LIEB: return std::sqrt(2.0);
    default: return 1.0;
    }
}

struct Cand {
    long long scan;   // position of this image in the reference's scan
    int tag;
    double angle;
};

}  // namespace

extern "C" int smd_geometry_info(int geom, int L, int *N, int *G, int *nsubs,
                                 int zn[3])
{
    Geo g;
    if (!geometry(geom, g) || L < 2) return SMD_EINVAL;
    if (L % 2) return SMD_EINVAL;                                   // subrouts.cpp:1119-1129
    if (geom != SMD_SQUARE && geom != SMD_LIEB && L % 3) return SMD_EINVAL;  // 1131-1139
    if (N) *N = g.nsubs * L * L;
    if (G) *G = g.grid_fac * L;
    if (nsubs) *nsubs = g.nsubs;
    if (zn) for (int s = 0; s < 3; s++) zn[s] = g.zn[s];
    return SMD_OK;
}

extern "C" int smd_build_lattice(int geom, int L, double *rvec, int *grid_map,
                                 int *nb1, int *nb2, int *nbx)
{
    Geo g;
    int N, G, ns, zn[3];
    if (smd_geometry_info(geom, L, &N, &G, &ns, zn) != SMD_OK) return SMD_EINVAL;
    geometry(geom, g);
    if (!rvec || !grid_map || !nb1 || !nb2 || !nbx) return SMD_EINVAL;
    const double a60 = kPi / 3.0, a90 = kPi / 2.0;
    const double c60 = std::cos(a60), s60 = std::sin(a60);
    const double av1[2] = {1.0, 0.0}, av2[2] = {c60, s60};
    const double szFac = size_factor(geom);
    const bool square_like = (geom == SMD_SQUARE || geom == SMD_LIEB);
    const double sq3 = std::sqrt(3.0);

    // ---- positions, site k = (i L + j) nsubs + sub (subrouts.cpp:2800-2895)
    int k = 0;
    for (int i = 0; i < L; i++) {
        for (int j = 0; j < L; j++) {
            double r0, r1;
            if (square_like) {
                r0 = i * szFac;
                r1 = j * szFac;
            } else {
                r0 = szFac * (i * av1[0] + j * av2[0]);
                r1 = szFac * (i * av1[1] + j * av2[1]);
            }
            if (ns == 1) {
                rvec[2 * k] = r0; rvec[2 * k + 1] = r1; k++;
            } else if (geom == SMD_HEXAGN) {
                rvec[2 * k] = r0 + 0.5 * sq3; rvec[2 * k + 1] = r1 + 0.5 * 1.0; k++;
                rvec[2 * k] = r0 + 1.0 * sq3; rvec[2 * k + 1] = r1 + 1.0 * 1.0; k++;
            } else {
                for (int n = 0; n < ns; n++) {
                    double ang = (geom == SMD_KAGOME) ? kPi - n * a60 : kPi - n * a90;
                    double amp = (geom == SMD_KAGOME) ? 1.0 : 0.5 * szFac;
                    if (geom == SMD_KAGOME) {
                        rvec[2 * k] = r0 + std::cos(ang);
                        rvec[2 * k + 1] = r1 + std::sin(ang);
                    } else {
                        rvec[2 * k] = r0 + amp * std::cos(ang);
                        rvec[2 * k + 1] = r1 + amp * std::sin(ang);
                    }
                    k++;
                }
            }
        }
    }

    // ---- grid map: invert the grid formula per site (subrouts.cpp:2903-2958)
    {
        const double fc = szFac / g.grid_fac;
        const int i0 = (geom == SMD_LIEB || geom == SMD_KAGOME) ? 1 : 0;
        for (int q = 0; q < G * G; q++) grid_map[q] = -1;
        int cnt = 0;
        for (int s = 0; s < N; s++) {
            double x = rvec[2 * s], y = rvec[2 * s + 1];
            long b, a;
            if (square_like) {
                a = std::lround(x / fc) + i0;
                b = std::lround(y / fc);
            } else {
                b = std::lround(y / (fc * s60));
                a = std::lround(x / fc - b * c60) + i0;
            }
            if (a < 0 || a >= G || b < 0 || b >= G) return SMD_EINVAL;
            double gx, gy;
            if (square_like) {
                gx = (a - i0) * fc;
                gy = b * fc;
            } else {
                gx = fc * ((a - i0) * av1[0] + b * av2[0]);
                gy = fc * ((a - i0) * av1[1] + b * av2[1]);
            }
            if (!(std::fabs(gx - x) < 1.0e-8 && std::fabs(gy - y) < 1.0e-8)) return SMD_EINVAL;
            grid_map[b + a * G] = s;
            cnt++;
        }
        if (cnt != N) return SMD_EINVAL;
    }

    // ---- neighbour tables (subrouts.cpp:2983-3316)
    const double spc = 500.0;
    const double a1[2] = {spc * av1[0], spc * av1[1]};
    const double a2[2] = {spc * av2[0], spc * av2[1]};
    std::vector<int> px(N), py(N);
    for (int s = 0; s < N; s++) {
        px[s] = (int)std::round(spc * rvec[2 * s]);
        py[s] = (int)std::round(spc * rvec[2 * s + 1]);
    }
    int nx1, nx2, ny;
    if (square_like) {
        nx1 = (int)std::round(L * szFac * spc);
        nx2 = (int)std::round(L * szFac * spc);
        ny = (int)std::round(L * szFac * spc);
    } else {
        nx1 = (int)std::round(L * szFac * a1[0]);
        nx2 = (int)std::round(L * szFac * a2[0]);
        ny = (int)std::round(L * szFac * (a1[1] + a2[1])) - 1;
    }
    // image 0 is the site itself; images 1..8 are the reference's shifts 0..7
    int sh[9][2] = {{0, 0}, {+nx1, 0}, {-nx1, 0}, {nx2, +ny}, {nx2, -ny},
                    {-nx2, +ny}, {-nx2, -ny}, {0, 0}, {0, 0}};
    if (square_like) {
        sh[7][0] = 0; sh[7][1] = +ny;
        sh[8][0] = 0; sh[8][1] = -ny;
    } else {
        sh[7][0] = +nx2 + nx1; sh[7][1] = +ny;
        sh[8][0] = -nx2 - nx1; sh[8][1] = -ny;
    }
    const int rA1 = (int)std::floor(spc * 1.10);
    const int rA3 = (int)std::floor(2.0 * spc * 1.05);
    const int rA2 = square_like ? (int)std::floor(std::sqrt(2.0) * spc * 1.05)
                                : (int)std::floor(std::sqrt(3.0) * spc * 1.05);
    const int R = 5;   // cell window: covers distance 2.1 for every geometry
    std::vector<Cand> l1, l2, l3;
    std::vector<int> seen(N, -1);
    int *tabs[3] = {nb1, nb2, nbx};
    for (int n = 0; n < N; n++) {
        const int cell = n / ns, ci = cell / L, cj = cell % L;
        l1.clear(); l2.clear(); l3.clear();
        for (int di = -R; di <= R; di++) {
            for (int dj = -R; dj <= R; dj++) {
                int ii = ((ci + di) % L + L) % L, jj = ((cj + dj) % L + L) % L;
                for (int sub = 0; sub < ns; sub++) {
                    int m = (ii * L + jj) * ns + sub;
                    if (m == n || seen[m] == n) continue;
                    seen[m] = n;
                    for (int im = 0; im < 9; im++) {
                        int dx = px[m] + sh[im][0] - px[n];
                        int dy = py[m] + sh[im][1] - py[n];
                        int dist = (int)std::floor(std::sqrt(std::pow(dx, 2) + std::pow(dy, 2)));
                        if (dist >= rA3 || dist == rA1 || dist == rA2) continue;
                        Cand c;
                        c.scan = (im == 0) ? m : (long long)N + 8LL * m + (im - 1);
                        c.tag = m;
                        c.angle = std::atan2(dy, dx);
                        if (dist < rA1) l1.push_back(c);
                        else if (dist < rA2) l2.push_back(c);
                        else l3.push_back(c);
                    }
                }
            }
        }
        if ((int)l1.size() != zn[0] || (int)l2.size() != zn[1] || (int)l3.size() != zn[2])
            return SMD_EINVAL;
        // kagome's average NN angle, summed in the reference's scan order
        double angle_sum = 0.0;
        if (geom == SMD_KAGOME) {
            std::vector<Cand> byscan(l1);
            std::sort(byscan.begin(), byscan.end(),
                      [](const Cand &a, const Cand &b) { return a.scan < b.scan; });
            for (const Cand &c : byscan) angle_sum += c.angle;
        }
        auto desc = [](const Cand &a, const Cand &b) { return a.angle > b.angle; };
        std::stable_sort(l1.begin(), l1.end(), desc);
        std::stable_sort(l2.begin(), l2.end(), desc);
        std::stable_sort(l3.begin(), l3.end(), desc);
        if (geom == SMD_HEXAGN) {
            std::rotate(l2.begin(), l2.begin() + ((n % 2 == 0) ? 1 : 2), l2.end());
        } else if (geom == SMD_KAGOME) {
            int ic1 = 1, ic2 = 1;
            double avg = angle_sum * (1.0 / (double)l1.size());
            if (avg > 0.0) {
                if (avg > 1.0) {
                    ic2 -= 1;
                } else {
                    ic1 -= 1;
                    ic2 -= 1;
                }
            }
            std::rotate(l1.begin(), l1.begin() + ic1, l1.end());
            std::rotate(l2.begin(), l2.begin() + ic2, l2.end());
        }
        std::vector<Cand> *lists[3] = {&l1, &l2, &l3};
        for (int s = 0; s < 3; s++)
            for (int q = 0; q < zn[s]; q++) tabs[s][n * zn[s] + q] = (*lists[s])[q].tag;
    }
    return SMD_OK;
}

extern "C" int smd_build_bonds(int N, const int zn[3], const int *nb1,
                               const int *nb2, const int *nbx, int j2_on,
                               int jx_on, int *bonds, int max_bonds,
                               int nbonds[4])
{
    // make_bondList (subrouts.cpp:3426-3570): a pair enters once, from the
    // first shell and site order that reaches it.  A hash set of pairs
    // stands in for the reference's N x N marker matrix.
    if (N <= 0 || !zn || !bonds || !nbonds) return SMD_EINVAL;
    const int *tab[3] = {nb1, nb2, nbx};
    const int on[3] = {1, j2_on, jx_on};
    std::unordered_set<long long> used;
    used.reserve((size_t)N * 8);
    int cnt = 0;
    for (int s = 0; s < 3; s++) {
        int before = cnt;
        if (on[s] && tab[s]) {
            for (int i = 0; i < N; i++) {
                for (int q = 0; q < zn[s]; q++) {
                    int j = tab[s][i * zn[s] + q];
                    if (j < 0) continue;
                    long long key = (long long)std::min(i, j) * N + std::max(i, j);
                    if (used.count(key)) continue;
                    if (cnt >= max_bonds) return SMD_EINVAL;
                    used.insert(key);
                    bonds[2 * cnt] = i;
                    bonds[2 * cnt + 1] = j;
                    cnt++;
                }
            }
        }
        nbonds[s + 1] = cnt - before;
    }
    nbonds[0] = cnt;
    return SMD_OK;
}

extern "C" int smd_window(const char *name, int n, double *w)
{
    // aux_code.cpp:249-435 (the window definitions), smd_code.cpp:2825-2894
    // (the names).  Coefficients are the published four- and five-term
    // cosine-sum windows the reference uses.
    if (!name || !w || n < 2) return SMD_EINVAL;
    const std::string s(name);
    const double two_pi = 2.0 * std::acos(-1.0);
    if (s == "nowin") {
        for (int i = 0; i < n; i++) w[i] = 1.0;
    } else if (s == "gauss") {
        const double dx = 2.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx - 1.0;
            w[i] = std::exp(-80.0 * std::pow(x, 2));
        }
    } else if (s == "ntall" || s == "black" || s == "flatw") {
        double c[5];
        if (s == "ntall") {
            const double v[5] = {0.3635819, 0.4891775, 0.1365995, 0.0106411, 0.0};
            std::memcpy(c, v, sizeof c);
        } else if (s == "black") {
            const double v[5] = {0.35875, 0.48829, 0.14128, 0.01168, 0.0};
            std::memcpy(c, v, sizeof c);
        } else {
            const double v[5] = {0.215578950, 0.416631580, 0.277263158, 0.083578947,
                                 0.006947368};
            std::memcpy(c, v, sizeof c);
        }
        const double dx = 1.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx;
            double r = (-c[1] * std::cos(1.0 * two_pi * x) + c[2] * std::cos(2.0 * two_pi * x) -
                        c[3] * std::cos(3.0 * two_pi * x));
            if (s == "flatw") r = r + c[4] * std::cos(4.0 * two_pi * x);
            w[i] = c[0] + r;
        }
    } else if (s == "lancz" || s == "sincw") {
        const bool lz = (s == "lancz");
        const double fc = lz ? 0.5 : 1.0;
        const double dx = 2.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = (i * dx - 1.0) * fc;
            double a = two_pi * x;
            double sinc = (a == 0.0) ? 1.0 : std::sin(a) / a;
            w[i] = (lz && std::fabs(x) > 0.5) ? 0.0 : sinc;
        }
    } else if (s == "hann1" || s == "hann2" || s == "hann3") {
        const int pw = s[4] - '0';
        const double dx = 1.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx;
            double r = 0.5 * (1.0 - std::cos(two_pi * x));
            w[i] = std::pow(r, pw);
        }
    } else {
        return SMD_EINVAL;
    }
    return SMD_OK;
}
