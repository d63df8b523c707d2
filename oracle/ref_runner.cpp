/*
 * ref_runner.cpp -- runs the reference's own SMD routines from their source
 * files, unchanged, as the parity pin for the oracle.  Test infrastructure:
 * only tests, the oracle fixture generator and the CPU baseline of bench.py
 * execute it.
 *
 * It compiles Codes_Folder/subrouts.cpp (which pulls in aux_code.cpp,
 * structures.cpp and the vendored dSFMT) against the stand-in MKL DFTI,
 * FFTW3 and GSL headers in oracle/shim/.  The reference's main program
 * (Codes_Folder/smd_code.cpp) needs MPI and is not built; this file repeats
 * the part of its main that the SMD path needs, calling the reference's own
 * functions for every computation:
 *   settings        convert_inputs2data       smd_code.cpp:472-666
 *   temperature     linear T grid             smd_code.cpp:834-881
 *   lattice         make_rvecList / make_nborsTable / make_bondList
 *                                             smd_code.cpp:1226-1870
 *   time grid       wmax, tmax, dwf           smd_code.cpp:2110-2114
 *   window          the named window builders smd_code.cpp:2808-2894
 *   sample loop     file read, checks, get_dynSpectrum, accumulation
 *                                             smd_code.cpp:3079-3291
 *
 *   static pre-pass (--prepass) local-field histograms and the capped
 *                   static structure factor of the samples, recorded as
 *                   locFieldHist and MCSamples_DFT_*Spec
 *                                                 smd_code.cpp:2289-2726
 *   output stage    (--outputs) sample averages, MC_Bin_SpecData, window
 *                   files, quantum-corrected zz spectra, centred slices, the
 *                   path and cut files            smd_code.cpp:2808-2983,
 *                                                 3596-3631, 3645-4130
 *
 * Usage: smd_ref_run WORKDIR SAMPLES_FILE FIRST COUNT [--dump-final]
 *        [--no-dwf-guard] [--outputs]
 * WORKDIR holds the six Settings_*.txt files and receives:
 *   ref_lattice.bin  tables built by the reference (layout below)
 *   ref_spec.bin     sum over the processed samples of Sqx/Sqy/Sqz rows
 *                    interleaved per q as in MC_Bin_SpecData
 *                    (smd_code.cpp:3613-3631), then the qSS sum
 *   ref_final.bin    final spin field of every processed sample (optional)
 * and prints one JSON line with the timing of the sample loop.
 */
#include <iomanip>
#include <iostream>
#include <stdio.h>
#include <fstream>
#include <sstream>
#include <complex>
#include <string>
#include <vector>
#include <chrono>
#include <limits>
#include <cmath>
#include <gsl/gsl_statistics.h>
#include <gsl/gsl_rng.h>
#include <experimental/filesystem>
#include <regex>
#include <algorithm>
#include <initializer_list>
#include <cstring>
#include <cctype>
#include <locale>
#include <sys/stat.h>
#include <unistd.h>
#include <mkl.h>
#include <fftw3.h>

using namespace std;
using namespace std::chrono;

namespace fs = experimental::filesystem;

#include "subrouts.cpp"

static bool read_words(const string &name, string *out, int n)
{
    ifstream f(name);
    if (!f.is_open()) return false;
    for (int i = 0; i < n; i++)
        if (!(f >> out[i])) return false;
    return true;
}

template <typename T>
static void put(ofstream &f, const T *p, size_t n)
{
    f.write(reinterpret_cast<const char *>(p), sizeof(T) * n);
}

int main(int argc, char **argv)
{
    if (argc < 5) {
        cerr << "usage: smd_ref_run WORKDIR SAMPLES FIRST COUNT"
                " [--dump-final] [--no-dwf-guard]\n";
        return 2;
    }
    const string workdir = argv[1];
    const string samples = argv[2];
    const long first = atol(argv[3]);
    const long count = atol(argv[4]);
    bool dump_final = false, dwf_guard = true, outputs = false, prepass = false, mc = false;
    long mc_therm = 0, mc_meas = 0;
    for (int a = 5; a < argc; a++) {
        string s = argv[a];
        if (s == "--dump-final") dump_final = true;
        if (s == "--no-dwf-guard") dwf_guard = false;
        if (s == "--outputs") outputs = true;
        if (s == "--prepass") prepass = true;
        if (s == "--mc" && a + 2 < argc) {
            mc = true;
            mc_therm = atol(argv[a + 1]);
            mc_meas = atol(argv[a + 2]);
            a += 2;
        }
    }
    if (chdir(workdir.c_str()) != 0) {
        cerr << "cannot enter " << workdir << "\n";
        return 2;
    }

    /* ---- code-execution flags (16 name/value pairs) */
    {
        ifstream f(fset0);
        string name;
        int val, vals[16];
        for (int i = 0; i < 16; i++) {
            if (!(f >> name >> val)) {
                cerr << "bad " << fset0 << "\n";
                return 3;
            }
            vals[i] = val;
        }
        ptON = vals[0]; ptAdapt = vals[1]; ptTrack = vals[2];
        ANNL_ON = vals[3]; FFTW_ON = vals[4]; RKCheck = vals[5];
        PBC_OFF = vals[6]; IsiModel = vals[7]; qcrystal = vals[8];
        with_recField = vals[9]; with_DFTcodes = vals[10];
        force_Stripes = vals[11]; refState_Zero = vals[12];
        qct_NeelPhase = vals[13]; qct_RemovePBC = vals[14];
        rec_orderMaps = vals[15];
    }
    if (qcrystal ? (qct_RemovePBC || !PBC_OFF) : (FFTW_ON || !with_DFTcodes)) {
        /* quasi-crystals: the reference's own check (smd_code.cpp:365-372) */
        cerr << "runner supports periodic crystals with with_DFTcodes=1, or"
                " quasi-crystals with PBC_OFF=1 and qct_RemovePBC=0\n";
        return 3;
    }

    /* ---- settings files */
    string in1[11], in2[8], in3[7], in4[7];
    if (!read_words(fset1, in1, 11) || !read_words(fset2, in2, 8) ||
        !read_words(fset3, in3, 7) || !read_words(fset4, in4, 7)) {
        cerr << "cannot read settings\n";
        return 3;
    }
    int inum = 0, flag = 0;
    convert_inputs2data(in1, in2, in3, in4, 0, inum, flag);
    if (flag > 0) {
        cerr << "invalid input " << inum << " in file " << flag << "\n";
        return 4;
    }
    npt = tpLstSz;
    double Temp = Temp1;
    if (npt > 1) Temp = Temp1 + tpIndex * (Temp2 - Temp1) / (npt - 1);

    dSFMT_init(20240601);

    /* ---- lattice */
    rvecList = Alloc_dble_array(Ns, 2);
    nbors1 = Alloc_intg_array(Ns, Zn1);
    nbors2 = Alloc_intg_array(Ns, Zn2);
    nborsX = Alloc_intg_array(Ns, ZnX);
    if (qcrystal) {
        /* tables read from outBin/ as smd_code.cpp:1248-1300 (sites) and
           1575-1660 (neighbours) read them, with their size checks and the
           reference's lattice-spacing check */
        ifstream st(outDir0 + "sitesList" + SzTag + ".bin", ios::binary | ios::ate);
        ifstream nb(outDir0 + "nborsList" + SzTag + ".bin", ios::binary | ios::ate);
        if (!st.is_open() || !nb.is_open() || (size_t)st.tellg() != (size_t)Ns * 2 * sizeof(double) ||
            (size_t)nb.tellg() != (size_t)Ns * (Zn1 + Zn2 + ZnX) * sizeof(int)) {
            cerr << "missing or invalid quasi-crystal tables\n";
            return 5;
        }
        st.seekg(0, ios::beg);
        nb.seekg(0, ios::beg);
        for (int k = 0; k < Ns; k++) st.read(reinterpret_cast<char *>(rvecList[k]), 2 * sizeof(double));
        for (int k = 0; k < Ns; k++) {
            nb.read(reinterpret_cast<char *>(nbors1[k]), Zn1 * sizeof(int));
            nb.read(reinterpret_cast<char *>(nbors2[k]), Zn2 * sizeof(int));
            nb.read(reinterpret_cast<char *>(nborsX[k]), ZnX * sizeof(int));
        }
        double lspc = 0.0;
        check_latticeSpc(lspc, flag);
        if (flag > 0) {
            cerr << "lattice spacing is not unit\n";
            return 5;
        }
    } else {
        if (multiSubs) r0List = Alloc_dble_array(Ns0, 2);
        dftGrid = Alloc_dble_array(Nsg, 2);
        gridMap = new int[Nsg];
        make_rvecList(flag);
        if (flag > 0) {
            cerr << "make_rvecList failed " << flag << "\n";
            return 5;
        }
        mkdir("outBin", 0755);
        make_nborsTable(flag);
        if (flag > 0) {
            cerr << "make_nborsTable failed " << flag << "\n";
            return 5;
        }
    }
    {
        int nbonds[4];
        vector<Point> ij;
        make_bondList(nbonds, ij);
        Nb1 = nbonds[1];
        Nb2 = nbonds[2];
        NbX = nbonds[3];
        Nb = Nb1 + Nb2 + NbX;
        bondList = new Point[Nb];
        zvalList = new Pts3d[Ns];
        for (int k = 0; k < Nb; k++) bondList[k] = ij[k];
        make_zvalList();
    }
    {
        ofstream f("ref_lattice.bin", ios::binary);
        int hdr[8] = {Ns, Zn1, Zn2, ZnX, Gsz, Nb1, Nb2, NbX};
        put(f, hdr, 8);
        for (int k = 0; k < Ns; k++) put(f, rvecList[k], 2);
        for (int k = 0; k < Ns; k++) put(f, nbors1[k], Zn1);
        for (int k = 0; k < Ns; k++) put(f, nbors2[k], Zn2);
        for (int k = 0; k < Ns; k++) put(f, nborsX[k], ZnX);
        if (qcrystal) {
            vector<int> none((size_t)Nsg, -1);   /* no DFT grid */
            put(f, none.data(), none.size());
        } else {
            put(f, gridMap, (size_t)Nsg);
        }
        for (int k = 0; k < Nb; k++) {
            int b[2] = {bondList[k].x, bondList[k].y};
            put(f, b, 2);
        }
    }

    /* ---- time grid and its guard */
    wmax = pi / dtm;
    tmax = ntm * dtm;
    dwf = 2.0 * pi / tmax;
    if (dwf_guard && dwf > dwf_min) {
        cerr << "dwf " << dwf << " exceeds dwf_min\n";
        return 6;
    }
    if (!qcrystal) {
        MKL_LONG dims[2] = {Gsz, Gsz};
        DftiCreateDescriptor(&handle, DFTI_DOUBLE, DFTI_COMPLEX, 2, dims);
        DftiCommitDescriptor(handle);
    } else if (prepass || outputs) {
        cerr << "--prepass and --outputs need a periodic crystal\n";
        return 3;
    }
    /* the direct-sum q spacing of a quasi-crystal (smd_code.cpp:1774) */
    if (qcrystal) dq = 4.0 * pi2 / Gsz;

    /* ---- temporal window */
    double *tmWinVec = new double[ntm];
    if (tWForm == "wread") {
        ifstream f("outBin/winvec.bin", ios::binary);
        f.read(reinterpret_cast<char *>(tmWinVec), ntm * sizeof(double));
        double mx = 0.0;
        for (int n = 0; n < ntm; n++) mx = max(mx, tmWinVec[n]);
        for (int n = 0; n < ntm; n++) tmWinVec[n] = (1.0 / mx) * tmWinVec[n];
    } else if (tWForm == "nowin") {
        for (int n = 0; n < ntm; n++) tmWinVec[n] = 1.0;
    } else if (tWForm == "gauss") {
        gaussWindow(ntm, tmWinVec);
    } else if (tWForm == "ntall") {
        blackNtWindow(ntm, tmWinVec);
    } else if (tWForm == "black") {
        blackHrWindow(ntm, tmWinVec);
    } else if (tWForm == "flatw") {
        flatTopWindow(ntm, tmWinVec);
    } else if (tWForm == "lancz") {
        lanczosWindow(ntm, 0.5, tmWinVec);
    } else if (tWForm == "sincw") {
        sincWindow(ntm, 1.0, tmWinVec);
    } else {
        int pw = 1;
        if (tWForm == "hann2") pw = 2;
        if (tWForm == "hann3") pw = 3;
        hannWindow(ntm, pw, tmWinVec);
    }

    if (mc) {
        /* The Monte Carlo stage of one rank (no tempering), as
           mc_hm_code.cpp:2797-2965 runs it: per MC step nmicro
           overrelaxation sweeps and ncanon heat-bath sweeps over shuffled
           site lists, then the total energy; from a disordered start
           (set_initialSpinField, IState high_T) with the reference's own
           generators (dSFMT seeded with 20240601 + FIRST, rand() seeded with
           FIRST for the shuffles).  Writes every step's total energy to
           ref_mc.bin (and a disordered lattice's impurity map to
           ref_imp.bin) and prints the mean energy per site of the last
           mc_meas steps. */
        dSFMT_init(20240601 + (int)first);   /* one stream per run */
        srand((unsigned)first);
        if (disOrder) {
            impField = new int[Ns];
            make_impurityField(impRatio, flag);
            ofstream fi("ref_imp.bin", ios::binary);
            put(fi, impField, (size_t)Ns);
        }
        double **spinField = Alloc_dble_array(Ns, 3);
        string info;
        set_initialSpinField(0, info, spinField);
        const double Beta = 1.0 / Temp;
        int *siteList = new int[Ns];
        Vec3d spinVec, spinVecNew, locField, unitVec;
        double RMat[9], EnrgTotal = 0.0, sum = 0.0;
        vector<double> trace;
        auto t1 = high_resolution_clock::now();
        for (long nmc = 0; nmc < mc_therm + mc_meas; nmc++) {
            for (int k = 0; k < nmicro; k++) {
                get_shuffledList(Ns, siteList);
                for (int n = 0; n < Ns; n++) {
                    const int i = siteList[n];
                    get_localSpin(i, spinField, spinVec);
                    get_localField(i, spinField, locField);
                    reflect_aboutVec(spinVec, locField, spinVecNew);
                    set_localSpin(i, spinVecNew, spinField);
                }
            }
            for (int k = 0; k < ncanon; k++) {
                get_shuffledList(Ns, siteList);
                for (int n = 0; n < Ns; n++) {
                    const int i = siteList[n];
                    get_localField(i, spinField, locField);
                    unitVec = normVec3d(locField);
                    get_rotZ2VMat(unitVec, RMat);
                    const double drand1 = dSFMT_getrnum();
                    const double drand2 = dSFMT_getrnum();
                    const double tht = 2.0 * pi * drand1;
                    double z = 0.0;
                    get_hBathSample(drand2, Beta, locField, z);
                    const double w = sqrt(1.0 - z * z);
                    spinVec[0] = w * cos(tht);
                    spinVec[1] = w * sin(tht);
                    spinVec[2] = z;
                    spinVecNew = MxVecProduct(RMat, spinVec);
                    set_localSpin(i, spinVecNew, spinField);
                }
            }
            get_energyValue(spinField, EnrgTotal);
            trace.push_back(EnrgTotal);
            if (nmc >= mc_therm) sum += EnrgTotal;
        }
        double ms = duration<double, milli>(high_resolution_clock::now() - t1).count();
        ofstream f("ref_mc.bin", ios::binary);
        put(f, trace.data(), trace.size());
        printf("{\"Ns\": %d, \"T\": %.10g, \"steps\": %ld, \"e_site\": %.17g, \"mc_ms\": %.3f}\n", Ns, Temp,
               mc_therm + mc_meas, mc_meas > 0 ? sum / mc_meas / Ns : 0.0, ms);
        return 0;
    }

    /* ---- sample file geometry (smd_code.cpp:976-1066) */
    const int PackSize = NMeas / crSkip;
    const size_t szIMap = (size_t)Ns * sizeof(int);
    const size_t szConf = (size_t)Ns * 3 * sizeof(double);
    const size_t szCPack = (disOrder ? szIMap : 0) + PackSize * szConf;
    ifstream fin(samples, ios::binary);
    if (!fin.is_open()) {
        cerr << "cannot open samples\n";
        return 7;
    }
    fin.seekg(0, ios::end);
    size_t szFile = (size_t)fin.tellg();
    const size_t szUnit = disOrder ? szCPack : szConf;
    if (szFile % szUnit != 0) {
        cerr << "samples file size " << szFile << " not a multiple of "
             << szUnit << "\n";
        return 7;
    }
    const long NSamps = disOrder ? (long)(szFile / szCPack) * PackSize
                                 : (long)(szFile / szConf);
    if (first < 0 || first + count > NSamps) {
        cerr << "sample range outside file (" << NSamps << ")\n";
        return 7;
    }

    double impRatioRef = 0.0;
    if (disOrder) {
        impField = new int[Ns];
        make_impurityField(impRatio, flag);
        impRatioRef = impurityRatio();
    }

    double **spinField = Alloc_dble_array(Ns, 3);
    if (prepass) {
        /* The static pre-pass of smd_code.cpp:2289-2726 over samples
           [first, first + count), calling the reference's functions. */
        ostringstream oss0;
        oss0 << fixed << setprecision(5) << Temp;
        const string tTagDat = "_T(" + oss0.str() + ")" + outLabel + ".dat";
        mkdir("outData", 0755);
        mkdir("outData/MC_Results", 0755);
        mkdir("outData/RK_Results", 0755);
        const int NHist = 201;
        const double hRange = 2.0 * maxLocField, boxSz = hRange / (NHist - 1), boxFc = 1.0 / boxSz;
        complex<double> *Sqx = new complex<double>[Nq], *Sqy = new complex<double>[Nq];
        complex<double> *Sqz = new complex<double>[Nq];
        double **specField = Alloc_dble_array(Nq, 3), **CMT_spcFd = Alloc_dble_array(Nq, 3);
        int **locFieldHist = Alloc_intg_array(NHist, 3);
        init_dble_array(CMT_spcFd, Nq, 3, 0.0);
        init_intg_array(locFieldHist, NHist, 3, 0);
        Vec3d locField;
        for (long s = first; s < first + count; s++) {
            long pack = s / PackSize, in_pack = s % PackSize;
            size_t base = pack * szCPack;
            if (disOrder) {
                fin.seekg(base, ios::beg);
                fin.read(reinterpret_cast<char *>(impField), szIMap);
                base += szIMap;
            }
            fin.seekg(base + in_pack * szConf, ios::beg);
            for (int k = 0; k < Ns; k++) fin.read(reinterpret_cast<char *>(spinField[k]), 3 * sizeof(double));
            for (int k = 0; k < Ns; k++) {
                get_localField(k, spinField, locField);
                locFieldHist[get_HistIndex(locField[0], maxLocField, boxFc, NHist)][0] += 1;
                locFieldHist[get_HistIndex(locField[1], maxLocField, boxFc, NHist)][1] += 1;
                locFieldHist[get_HistIndex(locField[2], maxLocField, boxFc, NHist)][2] += 1;
            }
            get_SqData_iMKL(spinField, Sqx, Sqy, Sqz);
            for (int k = 0; k < Nq; k++) {
                const double rx = abs(Sqx[k]), ry = abs(Sqy[k]), rz = abs(Sqz[k]);
                Sqx[k] = min(spec0Max, rx) * Sqx[k] / rx;
                Sqy[k] = min(spec0Max, ry) * Sqy[k] / ry;
                Sqz[k] = min(spec0Max, rz) * Sqz[k] / rz;
            }
            get_StaticSFac(Sqx, Sqy, Sqz, specField);
            for (int k = 0; k < Nq; k++)
                for (int m = 0; m < 3; m++) CMT_spcFd[k][m] += specField[k][m];
        }
        const double fcs = 1.0 / max(count - 1, 1L);
        for (int k = 0; k < Nq; k++)
            for (int m = 0; m < 3; m++) specField[k][m] = fcs * CMT_spcFd[k][m];
        double **xyA = Alloc_dble_array(Gsz, Gsz), **yzA = Alloc_dble_array(Gsz, Gsz);
        double **zzA = Alloc_dble_array(Gsz, Gsz), **ttA = Alloc_dble_array(Gsz, Gsz);
        dq = pi2 / Gsz;
        get_OrderedSpecArray2D(specField, xyA, yzA, zzA, ttA);
        record_SpecArray2D(xyA, "MCSamples_DFT_xySpec" + tTagDat, 1);
        record_SpecArray2D(yzA, "MCSamples_DFT_yzSpec" + tTagDat, 1);
        record_SpecArray2D(zzA, "MCSamples_DFT_zzSpec" + tTagDat, 1);
        record_SpecArray2D(ttA, "MCSamples_DFT_ttSpec" + tTagDat, 1);
        double histNorm[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < NHist; k++)
            for (int n = 0; n < 3; n++) histNorm[n] += locFieldHist[k][n];
        ofstream recHist(outDir1 + subDir1 + "locFieldHist" + tTagDat);
        for (int k = 0; k < NHist; k++) {
            recHist << fmtDbleFix(k * boxSz - maxLocField, 4, 8) << X2;
            for (int n = 0; n < 3; n++) recHist << fmtDbleFix(locFieldHist[k][n] / histNorm[n], 4, 10) << X2;
            recHist << endl;
        }
    }
    double **SqxWVec = Alloc_dble_array(Nq, ntm);
    double **SqyWVec = Alloc_dble_array(Nq, ntm);
    double **SqzWVec = Alloc_dble_array(Nq, ntm);
    double *qSStVec = new double[ntm];
    vector<double> accx((size_t)Nq * ntm, 0.0), accy(accx), accz(accx);
    vector<double> accq(ntm, 0.0);
    ofstream ffinal;
    if (dump_final) ffinal.open("ref_final.bin", ios::binary);

    auto t1 = high_resolution_clock::now();
    for (long s = first; s < first + count; s++) {
        long pack = s / PackSize, in_pack = s % PackSize;
        size_t base = pack * szCPack;
        if (disOrder) {
            fin.seekg(base, ios::beg);
            fin.read(reinterpret_cast<char *>(impField), szIMap);
            if (impurityRatio() != impRatioRef) {
                cerr << "impurity ratio check failed at sample " << s << "\n";
                return 8;
            }
            base += szIMap;
        }
        fin.seekg(base + in_pack * szConf, ios::beg);
        for (int k = 0; k < Ns; k++)
            fin.read(reinterpret_cast<char *>(spinField[k]), 3 * sizeof(double));
        if (fieldNorm(spinField) > 1.0) {
            cerr << "invalid spin field at sample " << s << "\n";
            return 8;
        }
        get_dynSpectrum(0, tmWinVec, spinField, SqxWVec, SqyWVec, SqzWVec,
                        qSStVec);
        for (int k = 0; k < Nq; k++)
            for (int n = 0; n < ntm; n++) {
                accx[(size_t)k * ntm + n] += SqxWVec[k][n];
                accy[(size_t)k * ntm + n] += SqyWVec[k][n];
                accz[(size_t)k * ntm + n] += SqzWVec[k][n];
            }
        for (int n = 0; n < ntm; n++) accq[n] += qSStVec[n];
        if (dump_final)
            for (int k = 0; k < Ns; k++) put(ffinal, spinField[k], 3);
    }
    auto t2 = high_resolution_clock::now();
    double ms = duration<double, milli>(t2 - t1).count();

    {
        ofstream f("ref_spec.bin", ios::binary);
        for (int k = 0; k < Nq; k++) {
            put(f, &accx[(size_t)k * ntm], ntm);
            put(f, &accy[(size_t)k * ntm], ntm);
            put(f, &accz[(size_t)k * ntm], ntm);
        }
        put(f, accq.data(), ntm);
    }
    if (outputs) {
        /* The root's output stage, calling the reference's own functions:
           sample averages (smd_code.cpp:3596-3611), their binary record
           (3613-3631), the window files (2895-2983), the quantum correction
           of the zz spectra (3645-3670; x and y are left as they are, the
           reference's xy/yz/tt values being undefined), centred slices
           (3813-3855), path and cut files (3700-3735, 3996-4130) and the
           autocorrelation (4019-4033). */
        ostringstream oss0;
        oss0 << fixed << setprecision(5) << Temp;
        const string tTagDat = "_T(" + oss0.str() + ")" + outLabel + ".dat";
        const string tTagBin = "_T(" + oss0.str() + ")" + outLabel + ".bin";
        mkdir("outData", 0755);
        mkdir("outData/RK_Check", 0755);
        mkdir("outData/MC_Results", 0755);
        mkdir("outData/RK_Results", 0755);
        const double fc = 1.0 / count;
        for (int k = 0; k < Nq; k++)
            for (int n = 0; n < ntm; n++) {
                SqxWVec[k][n] = fc * accx[(size_t)k * ntm + n];
                SqyWVec[k][n] = fc * accy[(size_t)k * ntm + n];
                SqzWVec[k][n] = fc * accz[(size_t)k * ntm + n];
            }
        for (int n = 0; n < ntm; n++) qSStVec[n] = fc * accq[n];
        {
            ofstream f(outDir0 + "MC_Bin_SpecData" + tTagBin, ios::binary);
            for (int k = 0; k < Nq; k++) {
                put(f, SqxWVec[k], ntm);
                put(f, SqyWVec[k], ntm);
                put(f, SqzWVec[k], ntm);
            }
            put(f, qSStVec, ntm);
        }
        {
            ofstream recWin1(outDir1 + "RK_Check/0WinTVec_" + tWForm + ".dat");
            ofstream recWin2(outDir1 + "RK_Check/0WinSpec_" + tWForm + ".dat");
            complex<double> *twvec = new complex<double>[ntm];
            prepare_wPlan_fftw1D();
            for (int n = 0; n < ntm; n++) twvec[n] = complex<double>(tmWinVec[n], 0.0);
            set_Input_fftw1D(twvec);
            double *wvec0 = new double[ntm], *wvec1 = new double[ntm];
            fftw_execute(wPlan);
            for (int n = 0; n < ntm; n++) {
                complex<double> wc(wfData[n][0], wfData[n][1]);
                wvec0[n] = (1.0 / ntm) * real(wc * conj(wc));
            }
            get_OrderedSpecArray1D(wvec0, wvec1);
            double wref = wvec1[0];
            for (int n = 1; n < ntm; n++)
                if (wvec1[n] > wref) wref = wvec1[n];
            const double fs0 = 2.0 / ntm;
            for (int n = 0; n < ntm; n++) {
                recWin1 << n * dtm << X3 << tmWinVec[n] << endl;
                recWin2 << n * fs0 - 1.0 << X3 << log10(wvec1[n] / wref) << endl;
            }
            destroy_wPlan_fftw1D();
            delete[] twvec;
            delete[] wvec0;
            delete[] wvec1;
        }
        /* dq and the path length npPath as main sets them
           (smd_code.cpp:1774-1791) */
        dq = pi2 / Gsz;
        {
            vector<Vec2d> bw;
            int n1 = 0;
            get_qPathWVectors(n1, bw);
            npPath = n1;
        }
        const double Beta = 1.0 / Temp;
        const double itFac = tmax / pi2;
        for (int k = 0; k < Nq; k++) {
            double qtFac = 1.0;
            for (int n = 0; n < ntm; n++) {
                const double wfreq = n * dwf, f2 = Beta * wfreq;
                if (n > 0) qtFac = f2 / (1.0 - exp(-f2));
                SqzWVec[k][n] = itFac * qtFac * SqzWVec[k][n];
            }
        }
        const int npw = ntm / 2, nmax = npw;
        double *zzSpecPath = new double[npPath];
        double **zzSpPathWVec = Alloc_dble_array(npPath, npw);
        double **specField = Alloc_dble_array(Nq, 3);
        double **xyA = Alloc_dble_array(Gsz, Gsz), **yzA = Alloc_dble_array(Gsz, Gsz);
        double **zzA = Alloc_dble_array(Gsz, Gsz), **ttA = Alloc_dble_array(Gsz, Gsz);
        const int nwSkip = ceil(0.1 * nmax);
        ostringstream wOss;
        for (int n = 0; n < npw; n++) {
            for (int k = 0; k < Nq; k++) {
                specField[k][0] = SqxWVec[k][n];
                specField[k][1] = SqyWVec[k][n];
                specField[k][2] = SqzWVec[k][n];
            }
            get_OrderedSpecArray2D(specField, xyA, yzA, zzA, ttA);
            get_Spec_qPath(zzA, zzSpecPath);
            for (int j = 0; j < npPath; j++) zzSpPathWVec[j][n] = zzSpecPath[j];
            if (n % nwSkip == 0) {
                wOss << fixed << setprecision(3) << n * dwf;
                record_SpecArray2D(zzA, "DFT_zzSpec_wfreq(" + wOss.str() + ")" + tTagDat, 1);
                wOss.str("");
            }
        }
        {
            ofstream f(outDir1 + subDir1 + "SpinSpin_Temporal_Corr" + tTagDat);
            for (int n = 0; n < ntm; n++)
                f << fmtDbleSci(n * dtm, 8, 15) << X4 << fmtDbleSci(qSStVec[n], 12, 22) << endl;
        }
        vector<Vec2d> bwvecPath;
        int n0 = 0;
        get_qPathWVectors(n0, bwvecPath);
        double *pathLPos = new double[npPath];
        {
            Vec2d wref = bwvecPath[0];
            double w0 = 0.0;
            for (int k = 0; k < npPath; k++) {
                Vec2d wvec = bwvecPath[k];
                const double qx = wvec[0] - wref[0], qy = wvec[1] - wref[1];
                w0 = w0 + sqrt(pow(qx, 2) + pow(qy, 2));
                pathLPos[k] = w0;
                wref = wvec;
            }
        }
        const bool sq = (geom == "square") || (geom == "lieb");
        const string p3 = (sq ? "YGMXG" : "KGMYG") + string("_wDepn_DFT_zzSpec") + tTagDat;
        const string p5 = (sq ? "YGMCut" : "KGMCut") + string("_wDepn_DFT_zzSpec") + tTagDat;
        const double cut1 = sq ? pi * 0.5 : 0.0, cut2 = sq ? pi * (1.0 + 0.5 * sq2) : pi;
        ofstream o3(outDir1 + subDir2 + p3), o5(outDir1 + subDir2 + p5);
        for (int k = 0; k < npPath; k++) {
            const double lpVal = pathLPos[k];
            for (int n = 0; n < nmax; n++) {
                const double wfreq = n * dwf, zzVal = zzSpPathWVec[k][n];
                o3 << fmtDbleSci(lpVal, 8, 15) << X4 << fmtDbleSci(wfreq, 8, 15) << X4
                   << fmtDbleSci(zzVal, 12, 22) << endl;
                if ((lpVal >= cut1) && (lpVal <= cut2))
                    o5 << fmtDbleSci(lpVal, 8, 15) << X4 << fmtDbleSci(wfreq, 8, 15) << X4
                       << fmtDbleSci(zzVal, 12, 22) << endl;
            }
            o3 << endl;
            o5 << endl;
        }
    }
    DftiFreeDescriptor(&handle);
    printf("{\"samples\": %ld, \"Ns\": %d, \"ntm\": %d, \"Nq\": %d, "
           "\"rk_loop_ms\": %.3f}\n",
           count, Ns, ntm, Nq, ms);
    return 0;
}
