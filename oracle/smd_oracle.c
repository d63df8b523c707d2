/*
 * smd_oracle.c -- CPU restatement of the reference's SMD path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path, never the
 * product.  Each function cites the reference lines it follows; the
 * restatement is pinned against the reference itself (oracle/_ref) through
 * the fixtures in tests/golden/.
 *
 * The dynamics restated here, per RK step (subrouts:11734-11902):
 *   ERef = E(S)
 *   K1 = dt h(S) x S,            P1 = S + K1/2
 *   K2 = dt h(P1) x P1,          P2 = S + K2/2
 *   K3 = dt h(P2) x P2,          P3 = S + K3
 *   K4 = dt h(P3) x P3
 *   S  = norm(S + (K1 + 2 K2 + 2 K3 + K4) / 6)
 *   sigma = sum_i |h_i(S) x S_i|^2,  scale = (ERef - E(S)) / sigma
 *   for i in order: S_i = norm(S_i + scale S_i x (h_i(S) x S_i)), with h_i
 *   read from the partially updated field (in place)
 * where h_i = -h z + sum_shells sum_nb J(a_i, a_nb) lambda_shell (.) S_nb.
 */
#include "smd_oracle.h"
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* constants as the reference defines them (subrouts:455-526) */
#define ORC_PI (acos(-1.0))

static double sq2(void) { return sqrt(2.0); }
static double sq3(void) { return sqrt(3.0); }

int orc_geometry(int geom, int L, int *N, int *G, int *nsubs, int zn[3])
{
    int ns, gf, z0, z1, z2;
    switch (geom) {
    case ORC_SQUARE: ns = 1; gf = 1; z0 = 4; z1 = 4; z2 = 4; break;
    case ORC_TRIANG: ns = 1; gf = 1; z0 = 6; z1 = 6; z2 = 6; break;
    case ORC_HEXAGN: ns = 2; gf = 3; z0 = 3; z1 = 6; z2 = 3; break;
    case ORC_KAGOME: ns = 3; gf = 2; z0 = 4; z1 = 4; z2 = 6; break;
    case ORC_LIEB:   ns = 2; gf = 2; z0 = 4; z1 = 4; z2 = 4; break;
    default: return 1;
    }
    *N = ns * L * L;
    *G = gf * L;
    *nsubs = ns;
    zn[0] = z0; zn[1] = z1; zn[2] = z2;
    return 0;
}

static double size_factor(int geom)
{
    /* make_rvecList / make_nborsTable size factors (subrouts:2728-2747) */
    switch (geom) {
    case ORC_HEXAGN: return sq3();
    case ORC_KAGOME: return 2.0;
    case ORC_LIEB: return sq2();
    default: return 1.0;
    }
}

typedef struct { int tag; double angle; } orc_nb;

static int cmp_angle_desc(const void *a, const void *b)
{
    double x = ((const orc_nb *)a)->angle, y = ((const orc_nb *)b)->angle;
    return (x > y) ? -1 : (x < y) ? 1 : 0;
}

static void rotate_left(orc_nb *v, int n, int k)
{
    if (n <= 0) return;
    k %= n;
    if (!k) return;
    orc_nb *tmp = (orc_nb *)malloc(sizeof(orc_nb) * n);
    for (int i = 0; i < n; i++) tmp[i] = v[(i + k) % n];
    memcpy(v, tmp, sizeof(orc_nb) * n);
    free(tmp);
}

int orc_make_lattice(int geom, int L, double *rvec, int *grid_map, int *nb1,
                     int *nb2, int *nbx)
{
    int N, G, nsubs, zn[3];
    if (orc_geometry(geom, L, &N, &G, &nsubs, zn)) return 1;
    const double pi = ORC_PI, a60 = pi / 3.0, a90 = pi / 2.0;
    const double c60 = cos(a60), s60 = sin(a60);
    const double av1[2] = {1.0, 0.0}, av2[2] = {c60, s60};
    const double szFac = size_factor(geom);
    const int square_like = (geom == ORC_SQUARE || geom == ORC_LIEB);

    /* ---- site positions, make_rvecList (subrouts:2714-2899) */
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
            if (geom == ORC_SQUARE || geom == ORC_TRIANG) {
                rvec[2 * k] = r0; rvec[2 * k + 1] = r1; k++;
            } else if (geom == ORC_HEXAGN) {
                rvec[2 * k] = r0 + 0.5 * sq3(); rvec[2 * k + 1] = r1 + 0.5 * 1.0; k++;
                rvec[2 * k] = r0 + 1.0 * sq3(); rvec[2 * k + 1] = r1 + 1.0 * 1.0; k++;
            } else if (geom == ORC_KAGOME) {
                for (int n = 0; n < nsubs; n++) {
                    double angle = pi - n * a60;
                    rvec[2 * k] = r0 + cos(angle);
                    rvec[2 * k + 1] = r1 + sin(angle);
                    k++;
                }
            } else {
                for (int n = 0; n < nsubs; n++) {
                    double angle = pi - n * a90;
                    rvec[2 * k] = r0 + 0.5 * szFac * cos(angle);
                    rvec[2 * k + 1] = r1 + 0.5 * szFac * sin(angle);
                    k++;
                }
            }
        }
    }
    if (k != N) return 1;

    /* ---- DFT grid and its map onto sites (subrouts:2903-2961) */
    {
        const double fc = szFac / (G / L);
        int i0 = (geom == ORC_LIEB || geom == ORC_KAGOME) ? 1 : 0;
        int cnt = 0;
        for (int i = 0; i < G; i++) {
            for (int j = 0; j < G; j++) {
                double x, y;
                if (square_like) {
                    x = (i - i0) * fc;
                    y = j * fc;
                } else {
                    x = fc * ((i - i0) * av1[0] + j * av2[0]);
                    y = fc * ((i - i0) * av1[1] + j * av2[1]);
                }
                int n = j + i * G;
                grid_map[n] = -1;
                for (int s = 0; s < N; s++) {
                    if (fabs(x - rvec[2 * s]) < 1.0e-8 &&
                        fabs(y - rvec[2 * s + 1]) < 1.0e-8) {
                        grid_map[n] = s;
                        cnt++;
                    }
                }
            }
        }
        if (cnt != N) return 2;
    }

    /* ---- neighbour tables, make_nborsTable (subrouts:2983-3316) */
    const double spc = 500.0;
    const double a1[2] = {spc * av1[0], spc * av1[1]};
    const double a2[2] = {spc * av2[0], spc * av2[1]};
    const long nplus = 9L * N;
    int *px = (int *)malloc(sizeof(int) * nplus);
    int *py = (int *)malloc(sizeof(int) * nplus);
    int *pz = (int *)malloc(sizeof(int) * nplus);
    for (int s = 0; s < N; s++) {
        px[s] = (int)round(spc * rvec[2 * s]);
        py[s] = (int)round(spc * rvec[2 * s + 1]);
        pz[s] = s;
    }
    int nx1, nx2, ny;
    if (square_like) {
        nx1 = (int)round(L * szFac * spc);
        nx2 = (int)round(L * szFac * spc);
        ny = (int)round(L * szFac * spc);
    } else {
        nx1 = (int)round(L * szFac * a1[0]);
        nx2 = (int)round(L * szFac * a2[0]);
        ny = (int)round(L * szFac * (a1[1] + a2[1])) - 1;
    }
    int sh[8][2] = {{+nx1, 0}, {-nx1, 0}, {nx2, +ny}, {nx2, -ny},
                    {-nx2, +ny}, {-nx2, -ny}, {0, 0}, {0, 0}};
    if (square_like) {
        sh[6][0] = 0; sh[6][1] = +ny;
        sh[7][0] = 0; sh[7][1] = -ny;
    } else {
        sh[6][0] = +nx2 + nx1; sh[6][1] = +ny;
        sh[7][0] = -nx2 - nx1; sh[7][1] = -ny;
    }
    long cntp = N;
    for (int s = 0; s < N; s++) {
        for (int m = 0; m < 8; m++) {
            px[cntp] = sh[m][0] + px[s];
            py[cntp] = sh[m][1] + py[s];
            pz[cntp] = s;
            cntp++;
        }
    }
    const int rA1 = (int)floor(spc * 1.10);
    const int rA3 = (int)floor(2.0 * spc * 1.05);
    const int rA2 = square_like ? (int)floor(sq2() * spc * 1.05)
                                : (int)floor(sq3() * spc * 1.05);
    orc_nb *l1 = (orc_nb *)malloc(sizeof(orc_nb) * nplus);
    orc_nb *l2 = (orc_nb *)malloc(sizeof(orc_nb) * nplus);
    orc_nb *l3 = (orc_nb *)malloc(sizeof(orc_nb) * nplus);
    int flag = 0;
    for (int n = 0; n < N && !flag; n++) {
        int nx = px[n], nyy = py[n], st = pz[n];
        int c1 = 0, c2 = 0, c3 = 0;
        double angle_sum = 0.0;
        for (long m = 0; m < nplus; m++) {
            if (pz[m] == st) continue;
            int n1 = px[m], n2 = py[m];
            int dist = (int)floor(sqrt(pow(n1 - nx, 2) + pow(n2 - nyy, 2)));
            double angle = atan2(n2 - nyy, n1 - nx);
            if (dist < rA1) {
                angle_sum += angle;
                l1[c1].tag = pz[m]; l1[c1].angle = angle; c1++;
            } else if (dist > rA1 && dist < rA2) {
                l2[c2].tag = pz[m]; l2[c2].angle = angle; c2++;
            } else if (dist > rA2 && dist < rA3) {
                l3[c3].tag = pz[m]; l3[c3].angle = angle; c3++;
            }
        }
        if (c1 != zn[0] || c2 != zn[1] || c3 != zn[2]) {
            flag = 2;
            break;
        }
        qsort(l1, c1, sizeof(orc_nb), cmp_angle_desc);
        qsort(l2, c2, sizeof(orc_nb), cmp_angle_desc);
        qsort(l3, c3, sizeof(orc_nb), cmp_angle_desc);
        if (geom == ORC_HEXAGN) {
            rotate_left(l2, c2, (st % 2 == 0) ? 1 : 2);
        } else if (geom == ORC_KAGOME) {
            int ic1 = 1, ic2 = 1;
            double avg = angle_sum * (1.0 / c1);
            if (avg > 0.0) {
                if (avg > 1.0) {
                    ic2 -= 1;
                } else {
                    ic1 -= 1;
                    ic2 -= 1;
                }
            }
            rotate_left(l1, c1, ic1);
            rotate_left(l2, c2, ic2);
        }
        for (int q = 0; q < c1; q++) nb1[st * zn[0] + q] = l1[q].tag;
        for (int q = 0; q < c2; q++) nb2[st * zn[1] + q] = l2[q].tag;
        for (int q = 0; q < c3; q++) nbx[st * zn[2] + q] = l3[q].tag;
    }
    free(px); free(py); free(pz);
    free(l1); free(l2); free(l3);
    return flag;
}

int orc_make_bonds(int N, const int zn[3], const int *nb1, const int *nb2,
                   const int *nbx, int j2_on, int jx_on, int *bonds,
                   int max_bonds, int nbonds[4])
{
    /* make_bondList (subrouts:3426-3570): a pair enters once, in the first
     * shell and site order that reaches it. */
    unsigned char *marker = (unsigned char *)malloc((size_t)N * N);
    memset(marker, 1, (size_t)N * N);
    const int *tab[3] = {nb1, nb2, nbx};
    const int on[3] = {1, j2_on, jx_on};
    int cnt = 0;
    for (int s = 0; s < 3; s++) {
        int before = cnt;
        if (on[s]) {
            for (int i = 0; i < N; i++) {
                for (int k = 0; k < zn[s]; k++) {
                    int j = tab[s][i * zn[s] + k];
                    if (j < 0) continue;
                    if (marker[(size_t)i * N + j]) {
                        if (cnt >= max_bonds) { free(marker); return -1; }
                        bonds[2 * cnt] = i;
                        bonds[2 * cnt + 1] = j;
                        cnt++;
                        marker[(size_t)i * N + j] = 0;
                        marker[(size_t)j * N + i] = 0;
                    }
                }
            }
        }
        nbonds[s + 1] = cnt - before;
    }
    nbonds[0] = cnt;
    free(marker);
    return 0;
}

void orc_local_field(const orc_model *m, int i, const double *S, double out[3])
{
    /* get_localField (subrouts:4465-4570) */
    out[0] = 0.0; out[1] = 0.0; out[2] = 0.0;
    if (fabs(m->h) > 1.0e-12) out[2] = -m->h;
    for (int s = 0; s < 3; s++) {
        if (!m->shell_on[s]) continue;
        for (int k = 0; k < m->zn[s]; k++) {
            int nb = m->nbr[s][i * m->zn[s] + k];
            if (nb < 0) continue;
            double J;
            if (m->disorder)
                J = m->J[s][m->imp[i]][m->imp[nb]];
            else
                J = m->J[s][0][0];
            if (s == 1 && m->lieb_delta_on)
                J += ((i & 1) ? -1 : 1) * ((k & 1) ? -1 : 1) * m->j2_delta;
            double Jv[3] = {J * m->lam[s][0], J * m->lam[s][1], J * m->lam[s][2]};
            for (int c = 0; c < 3; c++) out[c] += Jv[c] * S[3 * nb + c];
        }
    }
}

double orc_energy(const orc_model *m, const double *S)
{
    /* get_energyValue (subrouts:5181-5302) */
    double E = 0.0;
    int start = 0;
    for (int s = 0; s < 3; s++) {
        int cnt = m->nbonds[s];
        if (m->shell_on[s]) {
            for (int b = start; b < start + cnt; b++) {
                int i = m->bonds[2 * b], j = m->bonds[2 * b + 1];
                double J = m->disorder ? m->J[s][m->imp[i]][m->imp[j]] : m->J[s][0][0];
                if (s == 1 && m->lieb_delta_on)
                    J += ((i & 1) ? -1 : 1) * ((j & 1) ? -1 : 1) * m->j2_delta;
                double Jv[3] = {J * m->lam[s][0], J * m->lam[s][1], J * m->lam[s][2]};
                E += Jv[0] * S[3 * i] * S[3 * j] + Jv[1] * S[3 * i + 1] * S[3 * j + 1] +
                     Jv[2] * S[3 * i + 2] * S[3 * j + 2];
            }
        }
        start += cnt;
    }
    if (fabs(m->h) > 1.0e-12)
        for (int i = 0; i < m->N; i++) E += (-m->h) * S[3 * i + 2];
    return E;
}

int orc_window(const char *name, int n, double *w)
{
    /* window builders (aux:249-435), selection as smd:2825-2894 */
    const double two_pi = 2.0 * acos(-1.0);
    if (!strcmp(name, "nowin")) {
        for (int i = 0; i < n; i++) w[i] = 1.0;
    } else if (!strcmp(name, "gauss")) {
        const double dx = 2.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx - 1.0;
            w[i] = exp(-80.0 * pow(x, 2));
        }
    } else if (!strcmp(name, "ntall") || !strcmp(name, "black")) {
        /* Blackman-Nuttall / Blackman-Harris four-term cosine sums */
        const int nut = !strcmp(name, "ntall");
        const double a0 = nut ? 0.3635819 : 0.35875, a1 = nut ? 0.4891775 : 0.48829;
        const double a2 = nut ? 0.1365995 : 0.14128, a3 = nut ? 0.0106411 : 0.01168;
        const double dx = 1.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx;
            double r = (-a1 * cos(1.0 * two_pi * x) + a2 * cos(2.0 * two_pi * x) -
                        a3 * cos(3.0 * two_pi * x));
            w[i] = a0 + r;
        }
    } else if (!strcmp(name, "flatw")) {
        const double a0 = 0.215578950, a1 = 0.416631580, a2 = 0.277263158;
        const double a3 = 0.083578947, a4 = 0.006947368;
        const double dx = 1.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx;
            double r = (-a1 * cos(1.0 * two_pi * x) + a2 * cos(2.0 * two_pi * x) -
                        a3 * cos(3.0 * two_pi * x) + a4 * cos(4.0 * two_pi * x));
            w[i] = a0 + r;
        }
    } else if (!strcmp(name, "lancz") || !strcmp(name, "sincw")) {
        const int lanczos = !strcmp(name, "lancz");
        const double fc = lanczos ? 0.5 : 1.0;
        const double dx = 2.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = (i * dx - 1.0) * fc;
            double a = two_pi * x;
            double sinc = (a == 0.0) ? 1.0 : sin(a) / a;
            w[i] = (lanczos && fabs(x) > 0.5) ? 0.0 : sinc;
        }
    } else if (!strncmp(name, "hann", 4) && (name[4] >= '1' && name[4] <= '3') &&
               name[5] == 0) {
        const int pw = name[4] - '0';
        const double dx = 1.0 / (n - 1.0);
        for (int i = 0; i < n; i++) {
            double x = i * dx;
            double r = 0.5 * (1.0 - cos(two_pi * x));
            w[i] = pow(r, pw);
        }
    } else {
        return 1;
    }
    return 0;
}

/* ----------------------------------------------------------------- RK */

static void cross(const double a[3], const double b[3], double c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

static void normalise(const double v[3], double out[3])
{
    double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int c = 0; c < 3; c++) out[c] = v[c] / n;
}

typedef struct {
    double *prev, *next, *K[4];
} rk_work;

/* One RK4 step (subrouts:11741-11857); K arrays hold dt * h x S. */
static void rk4_step(const orc_model *m, double dt, double *S, rk_work *w)
{
    const int N = m->N;
    const double c[3] = {0.5, 0.5, 1.0};
    memcpy(w->prev, S, sizeof(double) * 3 * N);
    for (int st = 0; st < 4; st++) {
        for (int i = 0; i < N; i++) {
            double h[3], P[3];
            orc_local_field(m, i, w->prev, h);
            cross(h, &w->prev[3 * i], P);
            for (int q = 0; q < 3; q++) w->K[st][3 * i + q] = dt * P[q];
            if (st < 3)
                for (int q = 0; q < 3; q++)
                    w->next[3 * i + q] = S[3 * i + q] + c[st] * w->K[st][3 * i + q];
        }
        if (st < 3) memcpy(w->prev, w->next, sizeof(double) * 3 * N);
    }
    const double f1 = 1.0 / 6.0, f2 = 2.0 / 6.0;
    for (int i = 0; i < N; i++) {
        double v[3];
        for (int q = 0; q < 3; q++) {
            double d = f1 * (w->K[0][3 * i + q] + w->K[3][3 * i + q]) +
                       f2 * (w->K[1][3 * i + q] + w->K[2][3 * i + q]);
            v[q] = S[3 * i + q] + d;
        }
        normalise(v, &S[3 * i]);
    }
}

/* Energy correction (subrouts:11862-11900), in place in site order. */
static void energy_fix(const orc_model *m, double Eref, double *S)
{
    const int N = m->N;
    double sigma = 0.0;
    for (int i = 0; i < N; i++) {
        double h[3], P[3];
        orc_local_field(m, i, S, h);
        cross(h, &S[3 * i], P);
        sigma += P[0] * P[0] + P[1] * P[1] + P[2] * P[2];
    }
    double E1 = orc_energy(m, S);
    double scale = (Eref - E1) / sigma;
    for (int i = 0; i < N; i++) {
        double h[3], P[3], D[3], v[3];
        orc_local_field(m, i, S, h);
        cross(h, &S[3 * i], P);
        cross(&S[3 * i], P, D);
        for (int q = 0; q < 3; q++) v[q] = S[3 * i + q] + scale * D[q];
        normalise(v, &S[3 * i]);
    }
}

static int alloc_work(rk_work *w, int N)
{
    w->prev = (double *)malloc(sizeof(double) * 3 * N);
    w->next = (double *)malloc(sizeof(double) * 3 * N);
    for (int s = 0; s < 4; s++) w->K[s] = (double *)malloc(sizeof(double) * 3 * N);
    return 0;
}

static void free_work(rk_work *w)
{
    free(w->prev);
    free(w->next);
    for (int s = 0; s < 4; s++) free(w->K[s]);
}

static void one_step(const orc_model *m, double dt, int n, int fix_every,
                     double E0, double *S, rk_work *w)
{
    if (fix_every <= 1) {
        double Eref = orc_energy(m, S);
        rk4_step(m, dt, S, w);
        energy_fix(m, Eref, S);
    } else {
        rk4_step(m, dt, S, w);
        if (n % fix_every == 0) energy_fix(m, E0, S);
    }
}

int orc_evolve(const orc_model *m, double dt, int nsteps, int fix_every,
               double *S, int every, double *traj)
{
    rk_work w;
    alloc_work(&w, m->N);
    const double E0 = orc_energy(m, S);
    int rec = 0;
    if (traj) memcpy(traj, S, sizeof(double) * 3 * m->N), rec = 1;
    for (int n = 1; n <= nsteps; n++) {
        one_step(m, dt, n, fix_every, E0, S, &w);
        if (traj && every > 0 && n % every == 0) {
            memcpy(traj + (size_t)rec * 3 * m->N, S, sizeof(double) * 3 * m->N);
            rec++;
        }
    }
    free_work(&w);
    return 0;
}

/* S(q) of one state: grid transform then the q list. out[3][Q][2]. */
static void project(const orc_model *m, const double *S, int G,
                    const int *grid_map, int n_list, const double *qlist,
                    const double *pos, double list_scale, double *out, int Q,
                    double *grid_buf)
{
    if (G > 0) {
        /* get_SqData_iMKL (subrouts:8330-8432) */
        const double fc = sqrt(1.0 / ((double)G * G));
        for (int c = 0; c < 3; c++) {
            for (int k = 0; k < G * G; k++) {
                int idx = grid_map[k];
                grid_buf[2 * k] = (idx < 0) ? 0.0 : S[3 * idx + c];
                grid_buf[2 * k + 1] = 0.0;
            }
            orc_fft2d(grid_buf, G, G, -1);
            for (int k = 0; k < G * G; k++) {
                out[2 * ((size_t)c * Q + k)] = fc * grid_buf[2 * k];
                out[2 * ((size_t)c * Q + k) + 1] = fc * grid_buf[2 * k + 1];
            }
        }
    }
    const int off = G * G;
    for (int l = 0; l < n_list; l++) {
        /* direct sum of get_qct_SqData (subrouts:8460-8525) */
        double sr[3] = {0, 0, 0}, si[3] = {0, 0, 0};
        for (int k = 0; k < m->N; k++) {
            double ph = -(qlist[2 * l] * pos[2 * k] + qlist[2 * l + 1] * pos[2 * k + 1]);
            double cr = cos(ph), ci = sin(ph);
            for (int c = 0; c < 3; c++) {
                sr[c] += S[3 * k + c] * cr;
                si[c] += S[3 * k + c] * ci;
            }
        }
        for (int c = 0; c < 3; c++) {
            out[2 * ((size_t)c * Q + off + l)] = list_scale * sr[c];
            out[2 * ((size_t)c * Q + off + l) + 1] = list_scale * si[c];
        }
    }
}

int orc_dyn_spectrum(const orc_model *m, double dt, int n_rec, int stride,
                     int fix_every, const double *win, double *S, int G,
                     const int *grid_map, int n_list, const double *qlist,
                     const double *pos, double list_scale, double *spec,
                     double *qss, double *series, double *energy)
{
    const int N = m->N;
    const int Q = (G > 0 ? G * G : 0) + n_list;
    if (n_rec < 1 || stride < 1 || Q < 1) return 1;
    double *ser = (double *)malloc(sizeof(double) * 2 * 3 * (size_t)Q * n_rec);
    double *snap = (double *)malloc(sizeof(double) * 2 * 3 * (size_t)Q);
    double *grid_buf = (double *)malloc(sizeof(double) * 2 * (size_t)(G > 0 ? G * G : 1));
    double *S0 = (double *)malloc(sizeof(double) * 3 * N);
    memcpy(S0, S, sizeof(double) * 3 * N);
    rk_work w;
    alloc_work(&w, N);
    const double E0 = orc_energy(m, S);

    for (int r = 0; r < n_rec; r++) {
        if (r > 0) {
            for (int s = 1; s <= stride; s++)
                one_step(m, dt, (r - 1) * stride + s, fix_every, E0, S, &w);
        }
        project(m, S, G, grid_map, n_list, qlist, pos, list_scale, snap, Q, grid_buf);
        for (int c = 0; c < 3; c++)
            for (int q = 0; q < Q; q++) {
                size_t o = ((size_t)c * Q + q) * n_rec + r;
                ser[2 * o] = snap[2 * ((size_t)c * Q + q)];
                ser[2 * o + 1] = snap[2 * ((size_t)c * Q + q) + 1];
            }
        if (r == 0) {
            qss[0] = 1.0;                                  /* subrouts:11668 */
        } else {
            double p = 0.0;                                /* subrouts:11895-11902 */
            for (int i = 0; i < N; i++)
                p += S0[3 * i] * S[3 * i] + S0[3 * i + 1] * S[3 * i + 1] +
                     S0[3 * i + 2] * S[3 * i + 2];
            qss[r] = (1.0 / N) * p;
        }
        if (energy) energy[r] = orc_energy(m, S);
    }
    if (series) memcpy(series, ser, sizeof(double) * 2 * 3 * (size_t)Q * n_rec);

    /* windowed time transform and |.|^2 / n_rec (subrouts:12062-12109) */
    double *x = (double *)malloc(sizeof(double) * 2 * n_rec);
    const double sfc = sqrt(1.0 / n_rec);
    for (int c = 0; c < 3; c++) {
        for (int q = 0; q < Q; q++) {
            size_t o = ((size_t)c * Q + q) * n_rec;
            for (int t = 0; t < n_rec; t++) {
                x[2 * t] = win[t] * ser[2 * (o + t)];
                x[2 * t + 1] = win[t] * ser[2 * (o + t) + 1];
            }
            orc_fft1d(x, n_rec, -1);
            for (int t = 0; t < n_rec; t++) {
                double cr = sfc * x[2 * t], ci = sfc * x[2 * t + 1];
                spec[o + t] = cr * cr + ci * ci;
            }
        }
    }
    free(x);
    free(ser);
    free(snap);
    free(grid_buf);
    free(S0);
    free_work(&w);
    return 0;
}
