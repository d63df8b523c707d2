/*
 * smd_oracle.h -- CPU restatement of the reference's SMD path in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the
 * checker.  The product library never links or calls it.
 *
 * Every function names the reference lines it restates (paths relative to
 * the reference project; subrouts = Codes_Folder/subrouts.cpp, smd =
 * Codes_Folder/smd_code.cpp, aux = Codes_Folder/aux_code.cpp).  The
 * restatement is pinned against the reference's own code, compiled from its
 * sources by oracle/Makefile into oracle/_ref/smd_ref_run, through the golden
 * fixtures in tests/golden/.
 */
#ifndef SMD_ORACLE_H
#define SMD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SQUARE = 0, ORC_TRIANG = 1, ORC_HEXAGN = 2, ORC_KAGOME = 3,
       ORC_LIEB = 4 };

/* Geometry constants of convert_inputs2data (subrouts:1028-1067, 1141-1154).
 * Returns 0, or 1 for an unknown geometry. */
int orc_geometry(int geom, int L, int *N, int *G, int *nsubs, int zn[3]);

/* Site positions, grid map and neighbour tables, restating make_rvecList
 * (subrouts:2714-2962) and make_nborsTable (subrouts:2983-3316).
 * rvec[N][2], grid_map[G*G], nb1[N][zn0], nb2[N][zn1], nbx[N][zn2].
 * Returns the reference's flag: 0 ok, 1 wrong site count, 2 grid mapping or
 * neighbour count failure. */
int orc_make_lattice(int geom, int L, double *rvec, int *grid_map, int *nb1,
                     int *nb2, int *nbx);

/* Bond list of make_bondList (subrouts:3426-3570).  bonds[max_bonds][2];
 * nbonds[0..3] = total, NN, NNN, Xth.  Returns -1 when max_bonds is too
 * small. */
int orc_make_bonds(int N, const int zn[3], const int *nb1, const int *nb2,
                   const int *nbx, int j2_on, int jx_on, int *bonds,
                   int max_bonds, int nbonds[4]);

typedef struct {
    int N;
    int zn[3];
    const int *nbr[3];   /* [N][zn[s]], entries < 0 are ghosts */
    int shell_on[3];     /* 1, J2_ON, JX_ON */
    int disorder;        /* disOrder */
    const int *imp;      /* [N] impurity flags when disorder */
    double J[3][2][2];   /* J1Mat, J2Mat, JXMat */
    double lam[3][3];    /* lambdaVec1..3 */
    int lieb_delta_on;   /* J2ab_ON */
    double j2_delta;     /* J2_delta */
    double h;            /* extH along z (dMag = 2) */
    int nbonds[3];       /* Nb1, Nb2, NbX */
    const int *bonds;    /* [Nb][2] */
} orc_model;

/* get_localField (subrouts:4465-4570). */
void orc_local_field(const orc_model *m, int i, const double *S, double out[3]);

/* get_energyValue (subrouts:5181-5302). */
double orc_energy(const orc_model *m, const double *S);

/* The window builders of aux:249-435 selected by name as in smd:2825-2894.
 * name: nowin gauss ntall black flatw lancz sincw hann1 hann2 hann3.
 * Returns 0, or 1 for an unknown name ("wread" is a file, not a formula). */
int orc_window(const char *name, int n, double *out);

/* One sample of get_dynSpectrum (subrouts:11547-12149) generalised by a
 * record stride and a correction period:
 *   records r = 0 .. n_rec-1 are taken at RK step r*stride (stride 1 and
 *   fix_every 1 are the reference exactly);
 *   fix_every = 1 applies the energy correction after every step against the
 *   energy at the start of the step (subrouts:11736, 11862-11902);
 *   fix_every = F > 1 applies it after every F-th step against the energy of
 *   the initial state.
 * Projection: if G > 0, the grid transform of get_SqData_iMKL
 * (subrouts:8330-8432) with scale 1/sqrt(G*G); then n_list arbitrary points
 * q = qlist[l] as the direct sum of get_qct_SqData (subrouts:8460-8525):
 * list_scale * sum_k S_k exp(-i q . pos_k).
 * Outputs (Q = G*G + n_list):
 *   spec[3][Q][n_rec]   |FFT_t(w * S(q,t))|^2 / n_rec   (subrouts:12062-12109)
 *   qss[n_rec]          qss[0] = 1, qss[r] = (1/N) sum_i S0_i . S_i(r)
 *   series[3][Q][n_rec][2]  S(q,t) before the window (optional, may be NULL)
 *   energy[n_rec]       energy at each record (optional, may be NULL)
 * S[N][3] is updated in place to the final state, as the reference does. */
int orc_dyn_spectrum(const orc_model *m, double dt, int n_rec, int stride,
                     int fix_every, const double *win, double *S, int G,
                     const int *grid_map, int n_list, const double *qlist,
                     const double *pos, double list_scale, double *spec,
                     double *qss, double *series, double *energy);

/* RK evolution only: nsteps steps with the reference's per-step correction;
 * traj[(nsteps/every)+1][N][3] receives the state every `every` steps
 * (traj may be NULL).  Returns 0. */
int orc_evolve(const orc_model *m, double dt, int nsteps, int fix_every,
               double *S, int every, double *traj);

#ifdef __cplusplus
}
#endif

#endif
