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
 * Usage: smd_ref_run WORKDIR SAMPLES_FILE FIRST COUNT [--dump-final]
 *        [--no-dwf-guard] [--threads-note N]
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
    bool dump_final = false, dwf_guard = true;
    for (int a = 5; a < argc; a++) {
        string s = argv[a];
        if (s == "--dump-final") dump_final = true;
        if (s == "--no-dwf-guard") dwf_guard = false;
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
    if (qcrystal || FFTW_ON || !with_DFTcodes) {
        cerr << "runner supports periodic crystals with with_DFTcodes=1\n";
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
    (void)Temp;

    dSFMT_init(20240601);

    /* ---- lattice */
    rvecList = Alloc_dble_array(Ns, 2);
    if (multiSubs) r0List = Alloc_dble_array(Ns0, 2);
    dftGrid = Alloc_dble_array(Nsg, 2);
    gridMap = new int[Nsg];
    make_rvecList(flag);
    if (flag > 0) {
        cerr << "make_rvecList failed " << flag << "\n";
        return 5;
    }
    nbors1 = Alloc_intg_array(Ns, Zn1);
    nbors2 = Alloc_intg_array(Ns, Zn2);
    nborsX = Alloc_intg_array(Ns, ZnX);
    mkdir("outBin", 0755);
    make_nborsTable(flag);
    if (flag > 0) {
        cerr << "make_nborsTable failed " << flag << "\n";
        return 5;
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
        put(f, gridMap, (size_t)Nsg);
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
    {
        MKL_LONG dims[2] = {Gsz, Gsz};
        DftiCreateDescriptor(&handle, DFTI_DOUBLE, DFTI_COMPLEX, 2, dims);
        DftiCommitDescriptor(handle);
    }

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
    DftiFreeDescriptor(&handle);
    printf("{\"samples\": %ld, \"Ns\": %d, \"ntm\": %d, \"Nq\": %d, "
           "\"rk_loop_ms\": %.3f}\n",
           count, Ns, ntm, Nq, ms);
    return 0;
}
