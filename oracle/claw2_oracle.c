/*
 * claw2_oracle.c -- TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline).
 *
 * A serial CPU restatement of the reference's 2D classic step, kept in the
 * reference's own loop order, slice order, accumulation order and
 * parenthesisation so that its results can stand in for the Fortran, which
 * cannot be compiled here (no Fortran compiler in the image).  Nothing in the
 * product (pyclaw_b200/) links or calls this file; only tests/, the smoke check
 * in __graft_entry__.py and bench.py's CPU-baseline / reference arms do.
 *
 * Build with strict IEEE double arithmetic and no FMA contraction
 * (-O2 -ffp-contract=off), as the reference's gfortran build on x86-64 does.
 *
 * What follows which reference lines:
 *   orc_step2       src/pyclaw/classic/step2.f90:57-248
 *   orc_step2ds     src/pyclaw/classic/step2ds.f90:55-255
 *   flux2           src/pyclaw/classic/flux2.f90:85-206
 *   limiter         src/pyclaw/classic/limiter.f90:34-58
 *   philim          src/pyclaw/classic/philim.f90:18-55
 *   rpn2_euler      development/rp_approaches/rpn2_euler_5wave.f:63-298
 *   rpt2_euler      development/rp_approaches/rpt2_euler_5wave.f:39-95
 *   rpn2/rpt2_psystem  the f-wave p-system of apps/psystem_2d (restated from
 *                   its equations; pinned by apps/psystem_2d/verify_gauge*.txt)
 *   orc_fill_bc     src/pyclaw/solver.py:299-434 (q) and :438-576 (aux)
 *   orc_evolve      src/pyclaw/solver.py:582-699 with classic/solver.py:100-151
 * The acoustics, variable-coefficient acoustics and shallow-water Riemann
 * solvers belong to the external clawpack.riemann package (unpinned version,
 * not present in the reference tree); they are derived here from the
 * eigen-decompositions of the linearised systems (LeVeque, Finite Volume
 * Methods for Hyperbolic Problems, 2002, sections 3.8, 9.8, 21.5-21.6 and the
 * Harten-Hyman transonic fix of 15.3.5, written in the same structure as the
 * in-tree Euler solver).  Their exact arithmetic is therefore this file's own
 * definition; the reference's golden files pin them only to the tolerances
 * its tests use, and shallow water has no golden file at all.
 *
 * Array conventions: every array keeps the Fortran shape and lower bounds of
 * the routine it restates, through the index macros defined near each
 * routine, e.g. q1d(m, 1-mbc:maxm+mbc) -> Q1D(m,i).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#include "../include/claw2.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API __attribute__((visibility("default")))

static double dmax1(double a, double b) { return a > b ? a : b; }
static double dmin1(double a, double b) { return a < b ? a : b; }

/* Per-slice context: Riemann-solver scalars plus the /comroe/-style arrays
 * through which rpn2 hands its Roe averages to rpt2 (rpn2_euler_5wave.f:47-52). */
typedef struct orc_ctx {
    const claw2_problem* p;
    int maxm;
    double* roe;   /* 7 arrays of (maxm + 2*mbc + 2) doubles, index offset mbc+1 */
} orc_ctx;

#define ROE(k, i) ctx->roe[(size_t)(k) * (size_t)(ctx->maxm + 2 * mbc + 2) + (size_t)((i) + mbc + 1)]
enum { R_U2V2 = 0, R_U, R_V, R_ENTH, R_A, R_G1A2, R_EUV };

/* slice-array index macros (Fortran lower bound 1-mbc) */
#define Q1D(a, m, i)      (a)[((m) - 1) + meqn * ((i) + mbc - 1)]
#define AUXS(a, m, i)     (a)[((m) - 1) + maux * ((i) + mbc - 1)]
#define WAVE(m, mw, i)    wave[((m) - 1) + meqn * (((mw) - 1) + mwaves * ((i) + mbc - 1))]
#define SPD(mw, i)        s[((mw) - 1) + mwaves * ((i) + mbc - 1)]

/* ===================================================================== */
/* Riemann solvers                                                        */
/* ===================================================================== */

/* Euler Roe solver with Harten-Hyman entropy fix:
 * development/rp_approaches/rpn2_euler_5wave.f:63-298.  tracer=1 is the
 * 5-equation solver; tracer=0 drops the tracer equation and wave. */
static void rpn2_euler(int ixy, int mx, int meqn, int mwaves, int mbc,
                       const double* ql, const double* qr, double* wave, double* s,
                       double* amdq, double* apdq, orc_ctx* ctx, int tracer)
{
    const double gamma = ctx->p->params[0], gamma1 = ctx->p->params[1];
    int mu, mv, i, m, mw;
    double delta[4];
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }

    for (i = 2 - mbc; i <= mx + mbc; i++) {                        /* :87-104 */
        double rhsqrtl = sqrt(Q1D(qr, 1, i - 1));
        double rhsqrtr = sqrt(Q1D(ql, 1, i));
        double pl = gamma1 * (Q1D(qr, 4, i - 1) - 0.5 * (Q1D(qr, 2, i - 1) * Q1D(qr, 2, i - 1) +
                     Q1D(qr, 3, i - 1) * Q1D(qr, 3, i - 1)) / Q1D(qr, 1, i - 1));
        double pr = gamma1 * (Q1D(ql, 4, i) - 0.5 * (Q1D(ql, 2, i) * Q1D(ql, 2, i) +
                     Q1D(ql, 3, i) * Q1D(ql, 3, i)) / Q1D(ql, 1, i));
        double rhsq2 = rhsqrtl + rhsqrtr;
        double u = (Q1D(qr, mu, i - 1) / rhsqrtl + Q1D(ql, mu, i) / rhsqrtr) / rhsq2;
        double v = (Q1D(qr, mv, i - 1) / rhsqrtl + Q1D(ql, mv, i) / rhsqrtr) / rhsq2;
        double enth = ((Q1D(qr, 4, i - 1) + pl) / rhsqrtl + (Q1D(ql, 4, i) + pr) / rhsqrtr) / rhsq2;
        double u2v2 = u * u + v * v;
        double a2 = gamma1 * (enth - .5 * u2v2);
        ROE(R_U, i) = u; ROE(R_V, i) = v; ROE(R_ENTH, i) = enth; ROE(R_U2V2, i) = u2v2;
        ROE(R_A, i) = sqrt(a2);
        ROE(R_G1A2, i) = gamma1 / a2;
        ROE(R_EUV, i) = enth - u2v2;
    }

    for (i = 2 - mbc; i <= mx + mbc; i++) {                        /* :110-165 */
        double u = ROE(R_U, i), v = ROE(R_V, i), a = ROE(R_A, i), enth = ROE(R_ENTH, i);
        double a1, a2, a3, a4;
        delta[0] = Q1D(ql, 1, i) - Q1D(qr, 1, i - 1);
        delta[1] = Q1D(ql, mu, i) - Q1D(qr, mu, i - 1);
        delta[2] = Q1D(ql, mv, i) - Q1D(qr, mv, i - 1);
        delta[3] = Q1D(ql, 4, i) - Q1D(qr, 4, i - 1);
        a3 = ROE(R_G1A2, i) * (ROE(R_EUV, i) * delta[0] + u * delta[1] + v * delta[2] - delta[3]);
        a2 = delta[2] - v * delta[0];
        a4 = (delta[1] + (a - u) * delta[0] - a * a3) / (2.0 * a);
        a1 = delta[0] - a3 - a4;

        WAVE(1, 1, i) = a1; WAVE(mu, 1, i) = a1 * (u - a); WAVE(mv, 1, i) = a1 * v;
        WAVE(4, 1, i) = a1 * (enth - u * a);
        SPD(1, i) = u - a;
        WAVE(1, 2, i) = 0.0; WAVE(mu, 2, i) = 0.0; WAVE(mv, 2, i) = a2; WAVE(4, 2, i) = a2 * v;
        SPD(2, i) = u;
        WAVE(1, 3, i) = a3; WAVE(mu, 3, i) = a3 * u; WAVE(mv, 3, i) = a3 * v;
        WAVE(4, 3, i) = a3 * 0.5 * ROE(R_U2V2, i);
        SPD(3, i) = u;
        WAVE(1, 4, i) = a4; WAVE(mu, 4, i) = a4 * (u + a); WAVE(mv, 4, i) = a4 * v;
        WAVE(4, 4, i) = a4 * (enth + u * a);
        SPD(4, i) = u + a;
        if (tracer) {
            WAVE(5, 1, i) = 0.0; WAVE(5, 2, i) = 0.0; WAVE(5, 3, i) = 0.0; WAVE(5, 4, i) = 0.0;
            WAVE(1, 5, i) = 0.0; WAVE(mu, 5, i) = 0.0; WAVE(mv, 5, i) = 0.0; WAVE(4, 5, i) = 0.0;
            WAVE(5, 5, i) = Q1D(ql, 5, i) - Q1D(qr, 5, i - 1);
            SPD(5, i) = u;
        }
    }

    /* entropy fix, :195-286 (efix = .true. in the reference) */
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double rhoim1 = Q1D(qr, 1, i - 1);
        double pim1 = gamma1 * (Q1D(qr, 4, i - 1) - 0.5 * (Q1D(qr, mu, i - 1) * Q1D(qr, mu, i - 1) +
                      Q1D(qr, mv, i - 1) * Q1D(qr, mv, i - 1)) / rhoim1);
        double cim1 = sqrt(gamma * pim1 / rhoim1);
        double s0 = Q1D(qr, mu, i - 1) / rhoim1 - cim1;
        double rho1, rhou1, rhov1, en1, p1, c1, s1, sfract;
        double rhoi, pi, ci, s3, rho2, rhou2, rhov2, en2, p2, c2, s2;
        if (s0 >= 0.0 && SPD(1, i) > 0.0) {
            for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = 0.0;
            continue;
        }
        rho1 = Q1D(qr, 1, i - 1) + WAVE(1, 1, i);
        rhou1 = Q1D(qr, mu, i - 1) + WAVE(mu, 1, i);
        rhov1 = Q1D(qr, mv, i - 1) + WAVE(mv, 1, i);
        en1 = Q1D(qr, 4, i - 1) + WAVE(4, 1, i);
        p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
        c1 = sqrt(gamma * p1 / rho1);
        s1 = rhou1 / rho1 - c1;
        if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - SPD(1, i)) / (s1 - s0);
        else if (SPD(1, i) < 0.0) sfract = SPD(1, i);
        else sfract = 0.0;
        for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = sfract * WAVE(m, 1, i);

        if (SPD(2, i) >= 0.0) continue;
        for (m = 1; m <= meqn; m++) {
            Q1D(amdq, m, i) = Q1D(amdq, m, i) + SPD(2, i) * WAVE(m, 2, i);
            Q1D(amdq, m, i) = Q1D(amdq, m, i) + SPD(3, i) * WAVE(m, 3, i);
            if (tracer) Q1D(amdq, m, i) = Q1D(amdq, m, i) + SPD(5, i) * WAVE(m, 5, i);
        }

        rhoi = Q1D(ql, 1, i);
        pi = gamma1 * (Q1D(ql, 4, i) - 0.5 * (Q1D(ql, mu, i) * Q1D(ql, mu, i) +
             Q1D(ql, mv, i) * Q1D(ql, mv, i)) / rhoi);
        ci = sqrt(gamma * pi / rhoi);
        s3 = Q1D(ql, mu, i) / rhoi + ci;
        rho2 = Q1D(ql, 1, i) - WAVE(1, 4, i);
        rhou2 = Q1D(ql, mu, i) - WAVE(mu, 4, i);
        rhov2 = Q1D(ql, mv, i) - WAVE(mv, 4, i);
        en2 = Q1D(ql, 4, i) - WAVE(4, 4, i);
        p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
        c2 = sqrt(gamma * p2 / rho2);
        s2 = rhou2 / rho2 + c2;
        if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - SPD(4, i)) / (s3 - s2);
        else if (SPD(4, i) < 0.0) sfract = SPD(4, i);
        else continue;
        for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = Q1D(amdq, m, i) + sfract * WAVE(m, 4, i);
    }

    for (m = 1; m <= meqn; m++)                                      /* :291-298 */
        for (i = 2 - mbc; i <= mx + mbc; i++) {
            double df = 0.0;
            for (mw = 1; mw <= mwaves; mw++) df = df + SPD(mw, i) * WAVE(m, mw, i);
            Q1D(apdq, m, i) = df - Q1D(amdq, m, i);
        }
}

/* Euler transverse solver: development/rp_approaches/rpt2_euler_5wave.f:39-95 */
static void rpt2_euler(int ixy, int mx, int meqn, int mbc, const double* asdq,
                       double* bmasdq, double* bpasdq, orc_ctx* ctx, int tracer)
{
    int mu, mv, i, m, mw;
    double waveb[5][4] = {{0}}, sb[4] = {0};
    int nwb = tracer ? 4 : 3;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double u = ROE(R_U, i), v = ROE(R_V, i), a = ROE(R_A, i), enth = ROE(R_ENTH, i);
        double a1, a2, a3, a4;
        a3 = ROE(R_G1A2, i) * (ROE(R_EUV, i) * Q1D(asdq, 1, i) + u * Q1D(asdq, mu, i) +
                                v * Q1D(asdq, mv, i) - Q1D(asdq, 4, i));
        a2 = Q1D(asdq, mu, i) - u * Q1D(asdq, 1, i);
        a4 = (Q1D(asdq, mv, i) + (a - v) * Q1D(asdq, 1, i) - a * a3) / (2.0 * a);
        a1 = Q1D(asdq, 1, i) - a3 - a4;

        waveb[0][0] = a1; waveb[mu - 1][0] = a1 * u; waveb[mv - 1][0] = a1 * (v - a);
        waveb[3][0] = a1 * (enth - v * a); sb[0] = v - a;
        waveb[0][1] = a3; waveb[mu - 1][1] = a3 * u + a2; waveb[mv - 1][1] = a3 * v;
        waveb[3][1] = a3 * 0.5 * ROE(R_U2V2, i) + a2 * u; sb[1] = v;
        waveb[0][2] = a4; waveb[mu - 1][2] = a4 * u; waveb[mv - 1][2] = a4 * (v + a);
        waveb[3][2] = a4 * (enth + v * a); sb[2] = v + a;
        if (tracer) {
            waveb[4][0] = 0.0; waveb[4][1] = 0.0; waveb[4][2] = 0.0;
            waveb[0][3] = 0.0; waveb[1][3] = 0.0; waveb[2][3] = 0.0; waveb[3][3] = 0.0;
            waveb[4][3] = Q1D(asdq, 5, i); sb[3] = v;
        }
        for (m = 1; m <= meqn; m++) {
            Q1D(bmasdq, m, i) = 0.0;
            Q1D(bpasdq, m, i) = 0.0;
            for (mw = 1; mw <= nwb; mw++) {
                Q1D(bmasdq, m, i) = Q1D(bmasdq, m, i) + dmin1(sb[mw - 1], 0.0) * waveb[m - 1][mw - 1];
                Q1D(bpasdq, m, i) = Q1D(bpasdq, m, i) + dmax1(sb[mw - 1], 0.0) * waveb[m - 1][mw - 1];
            }
        }
    }
}

/* Constant-coefficient acoustics, q = (p, u, v).  Waves are the eigenvectors
 * (-Z,1,0) with speed -c and (Z,1,0) with speed +c of the normal system
 * (LeVeque 2002, sec. 3.8 / 18.4).  params: rho, bulk, cc, zz. */
static void rpn2_acoustics(int ixy, int mx, int meqn, int mwaves, int mbc,
                           const double* ql, const double* qr, double* wave, double* s,
                           double* amdq, double* apdq, orc_ctx* ctx)
{
    const double cc = ctx->p->params[2], zz = ctx->p->params[3];
    int mu, mv, i, m;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double delta1 = Q1D(ql, 1, i) - Q1D(qr, 1, i - 1);
        double delta2 = Q1D(ql, mu, i) - Q1D(qr, mu, i - 1);
        double a1 = (-delta1 + zz * delta2) / (2.0 * zz);
        double a2 = (delta1 + zz * delta2) / (2.0 * zz);
        WAVE(1, 1, i) = -a1 * zz; WAVE(mu, 1, i) = a1; WAVE(mv, 1, i) = 0.0; SPD(1, i) = -cc;
        WAVE(1, 2, i) = a2 * zz;  WAVE(mu, 2, i) = a2; WAVE(mv, 2, i) = 0.0; SPD(2, i) = cc;
        for (m = 1; m <= meqn; m++) {
            Q1D(amdq, m, i) = SPD(1, i) * WAVE(m, 1, i);
            Q1D(apdq, m, i) = SPD(2, i) * WAVE(m, 2, i);
        }
    }
}

/* Transverse split of asdq for constant acoustics: eigenvectors (-Z,0,1)
 * (speed -c) and (Z,0,1) (speed +c) of the transverse system. */
static void rpt2_acoustics(int ixy, int mx, int meqn, int mbc, const double* asdq,
                           double* bmasdq, double* bpasdq, orc_ctx* ctx)
{
    const double cc = ctx->p->params[2], zz = ctx->p->params[3];
    int mu, mv, i;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double a1 = (-Q1D(asdq, 1, i) + zz * Q1D(asdq, mv, i)) / (2.0 * zz);
        double a2 = (Q1D(asdq, 1, i) + zz * Q1D(asdq, mv, i)) / (2.0 * zz);
        Q1D(bmasdq, 1, i) = cc * a1 * zz; Q1D(bmasdq, mu, i) = 0.0; Q1D(bmasdq, mv, i) = -cc * a1;
        Q1D(bpasdq, 1, i) = cc * a2 * zz; Q1D(bpasdq, mu, i) = 0.0; Q1D(bpasdq, mv, i) = cc * a2;
    }
}

/* Variable-coefficient acoustics, aux = (rho, c).  Left-going wave in the
 * left cell's material, right-going wave in the right cell's (LeVeque 2002,
 * sec. 9.8 / 21.5). */
static void rpn2_vc_acoustics(int ixy, int mx, int meqn, int mwaves, int mbc, int maux,
                              const double* ql, const double* qr, const double* auxl,
                              const double* auxr, double* wave, double* s,
                              double* amdq, double* apdq)
{
    int mu, mv, i, m;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double zi = AUXS(auxl, 1, i) * AUXS(auxl, 2, i);
        double zim = AUXS(auxr, 1, i - 1) * AUXS(auxr, 2, i - 1);
        double delta1 = Q1D(ql, 1, i) - Q1D(qr, 1, i - 1);
        double delta2 = Q1D(ql, mu, i) - Q1D(qr, mu, i - 1);
        double a1 = (-delta1 + zi * delta2) / (zim + zi);
        double a2 = (delta1 + zim * delta2) / (zim + zi);
        WAVE(1, 1, i) = -a1 * zim; WAVE(mu, 1, i) = a1; WAVE(mv, 1, i) = 0.0;
        SPD(1, i) = -AUXS(auxr, 2, i - 1);
        WAVE(1, 2, i) = a2 * zi; WAVE(mu, 2, i) = a2; WAVE(mv, 2, i) = 0.0;
        SPD(2, i) = AUXS(auxl, 2, i);
        for (m = 1; m <= meqn; m++) {
            Q1D(amdq, m, i) = SPD(1, i) * WAVE(m, 1, i);
            Q1D(apdq, m, i) = SPD(2, i) * WAVE(m, 2, i);
        }
    }
}

/* Transverse vc-acoustics: asdq sits in cell i1 = i-2+ilr; the down-going
 * part uses the material below (aux1), the up-going part the material above
 * (aux3). */
static void rpt2_vc_acoustics(int ixy, int mx, int meqn, int mbc, int maux, int ilr,
                              const double* aux1, const double* aux2, const double* aux3,
                              const double* asdq, double* bmasdq, double* bpasdq)
{
    int mu, mv, i;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        int i1 = i - 2 + ilr;
        double cm = AUXS(aux1, 2, i1), cp = AUXS(aux3, 2, i1);
        double zm = AUXS(aux1, 1, i1) * AUXS(aux1, 2, i1);
        double zz = AUXS(aux2, 1, i1) * AUXS(aux2, 2, i1);
        double zp = AUXS(aux3, 1, i1) * AUXS(aux3, 2, i1);
        double a1 = (-Q1D(asdq, 1, i) + zz * Q1D(asdq, mv, i)) / (zm + zz);
        double a2 = (Q1D(asdq, 1, i) + zz * Q1D(asdq, mv, i)) / (zz + zp);
        Q1D(bmasdq, 1, i) = cm * a1 * zm; Q1D(bmasdq, mu, i) = 0.0; Q1D(bmasdq, mv, i) = -cm * a1;
        Q1D(bpasdq, 1, i) = cp * a2 * zp; Q1D(bpasdq, mu, i) = 0.0; Q1D(bpasdq, mv, i) = cp * a2;
    }
}

/* Shallow water Roe solver with a Harten-Hyman transonic fix, q = (h,hu,hv),
 * written in the structure of the in-tree Euler solver.  Roe averages:
 * h = (hl+hr)/2, u,v sqrt(h)-weighted, c = sqrt(g h) (LeVeque 2002, 15.3.3 and
 * 21.6).  The averages go to the transverse solver through ROE(). */
static void rpn2_shallow(int ixy, int mx, int meqn, int mwaves, int mbc,
                         const double* ql, const double* qr, double* wave, double* s,
                         double* amdq, double* apdq, orc_ctx* ctx)
{
    const double grav = ctx->p->params[0];
    int mu, mv, i, m, mw;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double hl = Q1D(qr, 1, i - 1), hr = Q1D(ql, 1, i);
        double hsqrtl = sqrt(hl), hsqrtr = sqrt(hr);
        double hsq2 = hsqrtl + hsqrtr;
        double ubar = (Q1D(qr, mu, i - 1) / hsqrtl + Q1D(ql, mu, i) / hsqrtr) / hsq2;
        double vbar = (Q1D(qr, mv, i - 1) / hsqrtl + Q1D(ql, mv, i) / hsqrtr) / hsq2;
        double hbar = 0.5 * (hl + hr);
        double cbar = sqrt(grav * hbar);
        double delta1 = hr - hl;
        double delta2 = Q1D(ql, mu, i) - Q1D(qr, mu, i - 1);
        double delta3 = Q1D(ql, mv, i) - Q1D(qr, mv, i - 1);
        double a1 = ((ubar + cbar) * delta1 - delta2) / (2.0 * cbar);
        double a2 = delta3 - vbar * delta1;
        double a3 = (delta2 - (ubar - cbar) * delta1) / (2.0 * cbar);
        ROE(R_U, i) = ubar; ROE(R_V, i) = vbar; ROE(R_A, i) = cbar;
        WAVE(1, 1, i) = a1; WAVE(mu, 1, i) = a1 * (ubar - cbar); WAVE(mv, 1, i) = a1 * vbar;
        SPD(1, i) = ubar - cbar;
        WAVE(1, 2, i) = 0.0; WAVE(mu, 2, i) = 0.0; WAVE(mv, 2, i) = a2;
        SPD(2, i) = ubar;
        WAVE(1, 3, i) = a3; WAVE(mu, 3, i) = a3 * (ubar + cbar); WAVE(mv, 3, i) = a3 * vbar;
        SPD(3, i) = ubar + cbar;
    }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double hl = Q1D(qr, 1, i - 1), hr = Q1D(ql, 1, i);
        double s0 = Q1D(qr, mu, i - 1) / hl - sqrt(grav * hl);
        double h1, hu1, s1, sfract, s3, h2, hu2, s2;
        if (s0 >= 0.0 && SPD(1, i) > 0.0) {
            for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = 0.0;
            continue;
        }
        h1 = hl + WAVE(1, 1, i);
        hu1 = Q1D(qr, mu, i - 1) + WAVE(mu, 1, i);
        s1 = hu1 / h1 - sqrt(grav * h1);
        if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - SPD(1, i)) / (s1 - s0);
        else if (SPD(1, i) < 0.0) sfract = SPD(1, i);
        else sfract = 0.0;
        for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = sfract * WAVE(m, 1, i);
        if (SPD(2, i) >= 0.0) continue;
        for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = Q1D(amdq, m, i) + SPD(2, i) * WAVE(m, 2, i);
        s3 = Q1D(ql, mu, i) / hr + sqrt(grav * hr);
        h2 = hr - WAVE(1, 3, i);
        hu2 = Q1D(ql, mu, i) - WAVE(mu, 3, i);
        s2 = hu2 / h2 + sqrt(grav * h2);
        if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - SPD(3, i)) / (s3 - s2);
        else if (SPD(3, i) < 0.0) sfract = SPD(3, i);
        else continue;
        for (m = 1; m <= meqn; m++) Q1D(amdq, m, i) = Q1D(amdq, m, i) + sfract * WAVE(m, 3, i);
    }
    for (m = 1; m <= meqn; m++)
        for (i = 2 - mbc; i <= mx + mbc; i++) {
            double df = 0.0;
            for (mw = 1; mw <= mwaves; mw++) df = df + SPD(mw, i) * WAVE(m, mw, i);
            Q1D(apdq, m, i) = df - Q1D(amdq, m, i);
        }
}

/* Transverse shallow water: eigenvectors (1,u,v-c), (0,1,0), (1,u,v+c) of the
 * transverse Roe matrix at the interface's Roe averages. */
static void rpt2_shallow(int ixy, int mx, int meqn, int mbc, const double* asdq,
                         double* bmasdq, double* bpasdq, orc_ctx* ctx)
{
    int mu, mv, i, m, mw;
    double waveb[3][3] = {{0}}, sb[3] = {0};
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double u = ROE(R_U, i), v = ROE(R_V, i), c = ROE(R_A, i);
        double a1 = ((v + c) * Q1D(asdq, 1, i) - Q1D(asdq, mv, i)) / (2.0 * c);
        double a2 = Q1D(asdq, mu, i) - u * Q1D(asdq, 1, i);
        double a3 = (Q1D(asdq, mv, i) - (v - c) * Q1D(asdq, 1, i)) / (2.0 * c);
        waveb[0][0] = a1; waveb[mu - 1][0] = a1 * u; waveb[mv - 1][0] = a1 * (v - c); sb[0] = v - c;
        waveb[0][1] = 0.0; waveb[mu - 1][1] = a2; waveb[mv - 1][1] = 0.0; sb[1] = v;
        waveb[0][2] = a3; waveb[mu - 1][2] = a3 * u; waveb[mv - 1][2] = a3 * (v + c); sb[2] = v + c;
        for (m = 1; m <= meqn; m++) {
            Q1D(bmasdq, m, i) = 0.0;
            Q1D(bpasdq, m, i) = 0.0;
            for (mw = 1; mw <= 3; mw++) {
                Q1D(bmasdq, m, i) = Q1D(bmasdq, m, i) + dmin1(sb[mw - 1], 0.0) * waveb[m - 1][mw - 1];
                Q1D(bpasdq, m, i) = Q1D(bpasdq, m, i) + dmax1(sb[mw - 1], 0.0) * waveb[m - 1][mw - 1];
            }
        }
    }
}

/* Two-dimensional p-system (nonlinear elasticity in layered media,
 * apps/psystem_2d/psystem.py): eps_t - u_x - v_y = 0, (rho u)_t - sigma_x = 0,
 * (rho v)_t - sigma_y = 0 with u = (rho u)/rho, aux = (rho, K, linearity, eps),
 * sigma = K eps (linearity 1) or exp(K eps) - 1 (linearity 2).  f-wave solver:
 * the flux jump f(q_i, x_i) - f(q_{i-1}, x_{i-1}), f = (-u, -sigma, 0) along the
 * normal, split on the eigenvectors (1, Z_{i-1}) with speed -c_{i-1} and
 * (1, -Z_i) with speed c_i, c = sqrt(sigma_eps / rho), Z = rho c (LeVeque 2002,
 * sec. 15.5 on f-waves; the same pairing of left and right materials as the
 * variable-coefficient acoustics solver). */
static void psys_cell(const double* aux, double eps, double* sigma, double* c, double* z)
{
    const double rho = aux[0], K = aux[1];
    double se;
    if (aux[2] == 1.0) { *sigma = K * eps; se = K; }
    else { const double e = exp(K * eps); *sigma = e - 1.0; se = K * e; }
    *c = sqrt(se / rho);
    *z = rho * *c;
}

static void rpn2_psystem(int ixy, int mx, int meqn, int mwaves, int mbc, int maux,
                         const double* ql, const double* qr, const double* auxl,
                         const double* auxr, double* wave, double* s,
                         double* amdq, double* apdq)
{
    int mu, mv, i, m;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        double sgl, cl, zl, sgr, cr, zr;
        psys_cell(&AUXS(auxr, 1, i - 1), Q1D(qr, 1, i - 1), &sgl, &cl, &zl);
        psys_cell(&AUXS(auxl, 1, i), Q1D(ql, 1, i), &sgr, &cr, &zr);
        const double ul = Q1D(qr, mu, i - 1) / AUXS(auxr, 1, i - 1);
        const double ur = Q1D(ql, mu, i) / AUXS(auxl, 1, i);
        const double df1 = (-ur) - (-ul);
        const double df2 = (-sgr) - (-sgl);
        const double b1 = (zr * df1 + df2) / (zl + zr);
        const double b2 = (zl * df1 - df2) / (zl + zr);
        WAVE(1, 1, i) = b1; WAVE(mu, 1, i) = b1 * zl; WAVE(mv, 1, i) = 0.0;
        SPD(1, i) = -cl;
        WAVE(1, 2, i) = b2; WAVE(mu, 2, i) = -b2 * zr; WAVE(mv, 2, i) = 0.0;
        SPD(2, i) = cr;
        for (m = 1; m <= meqn; m++) {
            Q1D(amdq, m, i) = WAVE(m, 1, i);
            Q1D(apdq, m, i) = WAVE(m, 2, i);
        }
    }
}

/* Transverse p-system: asdq sits in cell i1 = i-2+ilr; it is split on the
 * eigenvectors of the cells across the slice, (1, Z_b) going down with speed
 * -c_b in the cell below and (1, -Z_a) going up with speed c_a in the cell
 * above, with eps of those cells from aux(4) (set from q before each step by
 * the application, apps/psystem_2d/psystem.py:87-90).  This split reproduces
 * the reference's gauge files (apps/psystem_2d/verify_gauge*.txt) to their
 * printed digits; pairing either part with the cell's own eigenvector does
 * not (3e-5 after one step). */
static void rpt2_psystem(int ixy, int mx, int meqn, int mbc, int maux, int ilr,
                         const double* aux1, const double* aux2, const double* aux3,
                         const double* asdq, double* bmasdq, double* bpasdq)
{
    int mu, mv, i;
    if (ixy == 1) { mu = 2; mv = 3; } else { mu = 3; mv = 2; }
    for (i = 2 - mbc; i <= mx + mbc; i++) {
        int i1 = i - 2 + ilr;
        double sgb, cb, zb, sga, ca, za;
        psys_cell(&AUXS(aux1, 1, i1), AUXS(aux1, 4, i1), &sgb, &cb, &zb);
        psys_cell(&AUXS(aux3, 1, i1), AUXS(aux3, 4, i1), &sga, &ca, &za);
        const double gb = (za * Q1D(asdq, 1, i) + Q1D(asdq, mv, i)) / (zb + za);
        const double ga = (zb * Q1D(asdq, 1, i) - Q1D(asdq, mv, i)) / (zb + za);
        Q1D(bmasdq, 1, i) = -cb * gb; Q1D(bmasdq, mu, i) = 0.0; Q1D(bmasdq, mv, i) = -cb * gb * zb;
        Q1D(bpasdq, 1, i) = ca * ga; Q1D(bpasdq, mu, i) = 0.0; Q1D(bpasdq, mv, i) = -ca * ga * za;
    }
}

static void call_rpn2(int ixy, int mx, int meqn, int mwaves, int mbc, int maux,
                      const double* q1d, const double* aux2, double* wave, double* s,
                      double* amdq, double* apdq, orc_ctx* ctx)
{
    switch (ctx->p->rp) {
    case CLAW2_RP_ACOUSTICS:    rpn2_acoustics(ixy, mx, meqn, mwaves, mbc, q1d, q1d, wave, s, amdq, apdq, ctx); break;
    case CLAW2_RP_VC_ACOUSTICS: rpn2_vc_acoustics(ixy, mx, meqn, mwaves, mbc, maux, q1d, q1d, aux2, aux2, wave, s, amdq, apdq); break;
    case CLAW2_RP_EULER_4WAVE:  rpn2_euler(ixy, mx, meqn, mwaves, mbc, q1d, q1d, wave, s, amdq, apdq, ctx, 0); break;
    case CLAW2_RP_EULER_5WAVE:  rpn2_euler(ixy, mx, meqn, mwaves, mbc, q1d, q1d, wave, s, amdq, apdq, ctx, 1); break;
    case CLAW2_RP_SHALLOW_ROE:  rpn2_shallow(ixy, mx, meqn, mwaves, mbc, q1d, q1d, wave, s, amdq, apdq, ctx); break;
    case CLAW2_RP_PSYSTEM:      rpn2_psystem(ixy, mx, meqn, mwaves, mbc, maux, q1d, q1d, aux2, aux2, wave, s, amdq, apdq); break;
    }
}

static void call_rpt2(int ixy, int mx, int meqn, int mbc, int maux, int ilr,
                      const double* aux1, const double* aux2, const double* aux3,
                      const double* asdq, double* bmasdq, double* bpasdq, orc_ctx* ctx)
{
    switch (ctx->p->rp) {
    case CLAW2_RP_ACOUSTICS:    rpt2_acoustics(ixy, mx, meqn, mbc, asdq, bmasdq, bpasdq, ctx); break;
    case CLAW2_RP_VC_ACOUSTICS: rpt2_vc_acoustics(ixy, mx, meqn, mbc, maux, ilr, aux1, aux2, aux3, asdq, bmasdq, bpasdq); break;
    case CLAW2_RP_EULER_4WAVE:  rpt2_euler(ixy, mx, meqn, mbc, asdq, bmasdq, bpasdq, ctx, 0); break;
    case CLAW2_RP_EULER_5WAVE:  rpt2_euler(ixy, mx, meqn, mbc, asdq, bmasdq, bpasdq, ctx, 1); break;
    case CLAW2_RP_SHALLOW_ROE:  rpt2_shallow(ixy, mx, meqn, mbc, asdq, bmasdq, bpasdq, ctx); break;
    case CLAW2_RP_PSYSTEM:      rpt2_psystem(ixy, mx, meqn, mbc, maux, ilr, aux1, aux2, aux3, asdq, bmasdq, bpasdq); break;
    }
}

/* ===================================================================== */
/* limiter / philim: limiter.f90:34-58, philim.f90:18-55                   */
/* ===================================================================== */
static double philim(double a, double b, int meth)
{
    double r = b / a;
    switch (meth) {
    case 2: return dmax1(0.0, dmax1(dmin1(1.0, 2.0 * r), dmin1(2.0, r)));
    case 3: return (r + fabs(r)) / (1.0 + fabs(r));
    case 4: { double c = (1.0 + r) / 2.0; return dmax1(0.0, dmin1(dmin1(c, 2.0), 2.0 * r)); }
    case 5: return r;
    default: /* the computed GOTO falls through to minmod for ids outside 1..5 */
        return dmax1(0.0, dmin1(1.0, r));
    }
}

static void limiter(int mx, int meqn, int mwaves, int mbc, double* wave, const double* s,
                    const int32_t* mthlim)
{
    int mw, i, m;
    for (mw = 1; mw <= mwaves; mw++) {
        double dotr = 0.0;
        if (mthlim[mw - 1] == 0) continue;
        for (i = 0; i <= mx + 1; i++) {
            double wnorm2 = 0.0, dotl = dotr, wlimitr;
            dotr = 0.0;
            for (m = 1; m <= meqn; m++) {
                wnorm2 = wnorm2 + WAVE(m, mw, i) * WAVE(m, mw, i);
                dotr = dotr + WAVE(m, mw, i) * WAVE(m, mw, i + 1);
            }
            if (i == 0) continue;
            if (wnorm2 == 0.0) continue;
            if (SPD(mw, i) > 0.0) wlimitr = philim(wnorm2, dotl, mthlim[mw - 1]);
            else wlimitr = philim(wnorm2, dotr, mthlim[mw - 1]);
            for (m = 1; m <= meqn; m++) WAVE(m, mw, i) = wlimitr * WAVE(m, mw, i);
        }
    }
}

/* ===================================================================== */
/* flux2: src/pyclaw/classic/flux2.f90:85-206                              */
/* ===================================================================== */
typedef struct orc_work {
    double *qadd, *fadd, *gadd, *q1d, *dtdx1d, *dtdy1d, *aux1, *aux2, *aux3;
    double *wave, *s, *amdq, *apdq, *cqxx, *bmasdq, *bpasdq, *roe;
} orc_work;

#define GADD(m, k, i) gadd[((m) - 1) + meqn * (((k) - 1) + 2 * ((i) + mbc - 1))]
#define DTDX1D(i) dtdx1d[(i) + mbc - 1]

static void flux2(int ixy, int mx, const claw2_problem* p, const double* q1d,
                  const double* dtdx1d, const double* aux1, const double* aux2,
                  const double* aux3, int method2, int method3, double* qadd,
                  double* fadd, double* gadd, double* cfl1d, orc_work* w, orc_ctx* ctx)
{
    const int meqn = p->num_eqn, mwaves = p->num_waves, maux = p->num_aux, mbc = p->num_ghost;
    double *wave = w->wave, *s = w->s, *amdq = w->amdq, *apdq = w->apdq, *cqxx = w->cqxx;
    double *bmasdq = w->bmasdq, *bpasdq = w->bpasdq;
    int limit = 0, mw, m, i;
    for (mw = 0; mw < mwaves; mw++) if (p->mthlim[mw] > 0) limit = 1;

    for (i = 1 - mbc; i <= mx + mbc; i++)
        for (m = 1; m <= meqn; m++) {
            Q1D(qadd, m, i) = 0.0; Q1D(fadd, m, i) = 0.0;
            GADD(m, 1, i) = 0.0; GADD(m, 2, i) = 0.0;
        }

    call_rpn2(ixy, mx, meqn, mwaves, mbc, maux, q1d, aux2, wave, s, amdq, apdq, ctx);

    /* forall statement 1 then forall statement 2 (:108-111) */
    for (i = 1; i <= mx + 1; i++)
        for (m = 1; m <= meqn; m++) Q1D(qadd, m, i) = Q1D(qadd, m, i) - DTDX1D(i) * Q1D(apdq, m, i);
    for (i = 1; i <= mx + 1; i++)
        for (m = 1; m <= meqn; m++) Q1D(qadd, m, i - 1) = Q1D(qadd, m, i - 1) - DTDX1D(i - 1) * Q1D(amdq, m, i);

    *cfl1d = 0.0;                                                   /* :114-122 */
    for (mw = 1; mw <= mwaves; mw++)
        for (i = 1; i <= mx + 1; i++)
            *cfl1d = dmax1(dmax1(*cfl1d, DTDX1D(i) * SPD(mw, i)), -DTDX1D(i - 1) * SPD(mw, i));

    if (method2 != 1) {
        if (limit) limiter(mx, meqn, mwaves, mbc, wave, s, p->mthlim);
        for (i = 2 - mbc; i <= mx + mbc; i++) {                      /* :137-163 */
            double dtdxave = 0.5 * (DTDX1D(i - 1) + DTDX1D(i));
            for (m = 1; m <= meqn; m++) {
                Q1D(cqxx, m, i) = 0.0;
                for (mw = 1; mw <= mwaves; mw++) {
                    double sw = p->use_fwave ? copysign(1.0, SPD(mw, i)) : fabs(SPD(mw, i));
                    Q1D(cqxx, m, i) = Q1D(cqxx, m, i) + sw * (1.0 - fabs(SPD(mw, i)) * dtdxave) * WAVE(m, mw, i);
                }
                Q1D(fadd, m, i) = Q1D(fadd, m, i) + 0.5 * Q1D(cqxx, m, i);
            }
        }
    }

    if (method3 <= 0) return;                                        /* :168 */
    if (method2 > 1 && method3 == 2) {
        for (i = 1; i <= mx + 1; i++)
            for (m = 1; m <= meqn; m++) {
                Q1D(amdq, m, i) = Q1D(amdq, m, i) + Q1D(cqxx, m, i);
                Q1D(apdq, m, i) = Q1D(apdq, m, i) - Q1D(cqxx, m, i);
            }
    }
    call_rpt2(ixy, mx, meqn, mbc, maux, 1, aux1, aux2, aux3, amdq, bmasdq, bpasdq, ctx);
    for (i = 1; i <= mx + 1; i++)
        for (m = 1; m <= meqn; m++) GADD(m, 1, i - 1) = GADD(m, 1, i - 1) - 0.5 * DTDX1D(i - 1) * Q1D(bmasdq, m, i);
    for (i = 1; i <= mx + 1; i++)
        for (m = 1; m <= meqn; m++) GADD(m, 2, i - 1) = GADD(m, 2, i - 1) - 0.5 * DTDX1D(i - 1) * Q1D(bpasdq, m, i);
    call_rpt2(ixy, mx, meqn, mbc, maux, 2, aux1, aux2, aux3, apdq, bmasdq, bpasdq, ctx);
    for (i = 1; i <= mx + 1; i++)
        for (m = 1; m <= meqn; m++) GADD(m, 1, i) = GADD(m, 1, i) - 0.5 * DTDX1D(i) * Q1D(bmasdq, m, i);
    for (i = 1; i <= mx + 1; i++)
        for (m = 1; m <= meqn; m++) GADD(m, 2, i) = GADD(m, 2, i) - 0.5 * DTDX1D(i) * Q1D(bpasdq, m, i);
}

/* ===================================================================== */
/* workspace                                                              */
/* ===================================================================== */
static int work_alloc(const claw2_problem* p, orc_work* w, orc_ctx* ctx)
{
    const int meqn = p->num_eqn, mwaves = p->num_waves, mbc = p->num_ghost;
    const int maux = p->num_aux > 0 ? p->num_aux : 1;
    const int maxm = p->mx > p->my ? p->mx : p->my;
    const size_t n = (size_t)maxm + 2 * (size_t)mbc;
    memset(w, 0, sizeof *w);
    w->qadd = calloc(meqn * n, sizeof(double));
    w->fadd = calloc(meqn * n, sizeof(double));
    w->gadd = calloc(2 * meqn * n, sizeof(double));
    w->q1d = calloc(meqn * n, sizeof(double));
    w->dtdx1d = calloc(n, sizeof(double));
    w->dtdy1d = calloc(n, sizeof(double));
    w->aux1 = calloc(maux * n, sizeof(double));
    w->aux2 = calloc(maux * n, sizeof(double));
    w->aux3 = calloc(maux * n, sizeof(double));
    w->wave = calloc(meqn * mwaves * n, sizeof(double));
    w->s = calloc(mwaves * n, sizeof(double));
    w->amdq = calloc(meqn * n, sizeof(double));
    w->apdq = calloc(meqn * n, sizeof(double));
    w->cqxx = calloc(meqn * n, sizeof(double));
    w->bmasdq = calloc(meqn * n, sizeof(double));
    w->bpasdq = calloc(meqn * n, sizeof(double));
    w->roe = calloc(7 * (n + 2), sizeof(double));
    ctx->p = p; ctx->maxm = maxm; ctx->roe = w->roe;
    if (!w->qadd || !w->fadd || !w->gadd || !w->q1d || !w->dtdx1d || !w->dtdy1d || !w->aux1 ||
        !w->aux2 || !w->aux3 || !w->wave || !w->s || !w->amdq || !w->apdq || !w->cqxx ||
        !w->bmasdq || !w->bpasdq || !w->roe)
        return CLAW2_ERR_NOMEM;
    return CLAW2_OK;
}

static void work_free(orc_work* w)
{
    free(w->qadd); free(w->fadd); free(w->gadd); free(w->q1d); free(w->dtdx1d); free(w->dtdy1d);
    free(w->aux1); free(w->aux2); free(w->aux3); free(w->wave); free(w->s); free(w->amdq);
    free(w->apdq); free(w->cqxx); free(w->bmasdq); free(w->bpasdq); free(w->roe);
}

/* 2D ghosted arrays, Fortran order: (m, 1-mbc:mx+mbc, 1-mbc:my+mbc) */
#define A2(a, nc, m, i, j) (a)[((m) - 1) + (nc) * (((i) + mbc - 1) + (size_t)(mx + 2 * mbc) * ((j) + mbc - 1))]

static int check_problem(const claw2_problem* p)
{
    int mw;
    if (!p || p->num_ghost != CLAW2_NUM_GHOST || p->mx < 1 || p->my < 1) return CLAW2_ERR_INVALID;
    if (p->num_eqn < 1 || p->num_eqn > CLAW2_MAX_EQN || p->num_waves < 1 || p->num_waves > CLAW2_MAX_WAVES)
        return CLAW2_ERR_INVALID;
    if (p->order < 1 || p->order > 2 || p->transverse < -1 || p->transverse > 2) return CLAW2_ERR_INVALID;
    for (mw = 0; mw < p->num_waves; mw++) if (p->mthlim[mw] < 0) return CLAW2_ERR_INVALID;
    switch (p->rp) {
    case CLAW2_RP_ACOUSTICS: if (p->num_eqn != 3 || p->num_waves != 2) return CLAW2_ERR_INVALID; break;
    case CLAW2_RP_VC_ACOUSTICS: if (p->num_eqn != 3 || p->num_waves != 2 || p->num_aux < 2) return CLAW2_ERR_INVALID; break;
    case CLAW2_RP_EULER_4WAVE: if (p->num_eqn != 4 || p->num_waves != 4) return CLAW2_ERR_INVALID; break;
    case CLAW2_RP_EULER_5WAVE: if (p->num_eqn != 5 || p->num_waves != 5) return CLAW2_ERR_INVALID; break;
    case CLAW2_RP_SHALLOW_ROE: if (p->num_eqn != 3 || p->num_waves != 3) return CLAW2_ERR_INVALID; break;
    case CLAW2_RP_PSYSTEM: if (p->num_eqn != 3 || p->num_waves != 2 || p->num_aux < 4) return CLAW2_ERR_INVALID; break;
    default: return CLAW2_ERR_INVALID;
    }
    if (p->index_capa >= p->num_aux) return CLAW2_ERR_INVALID;
    return CLAW2_OK;
}

/* ===================================================================== */
/* step2: src/pyclaw/classic/step2.f90:57-248                              */
/* ===================================================================== */
ORC_API int orc_step2(const claw2_problem* p, const double* qold, double* qnew,
                      const double* aux, double dt, double* cfl_out)
{
    const int meqn = p->num_eqn, mbc = p->num_ghost, mx = p->mx, my = p->my;
    const int maux = p->num_aux, index_capa = p->index_capa + 1;
    orc_work w; orc_ctx ctx;
    double cfl = 0.0, cfl1d, dtdx, dtdy;
    int i, j, m, ma, rc = check_problem(p);
    if (rc) return rc;
    if (p->transverse < 0) return CLAW2_ERR_INVALID;
    if ((rc = work_alloc(p, &w, &ctx))) { work_free(&w); return rc; }
    {
        double *q1d = w.q1d, *qadd = w.qadd, *fadd = w.fadd, *gadd = w.gadd;
        double *dtdx1d = w.dtdx1d, *dtdy1d = w.dtdy1d;
        const int maxm = ctx.maxm;
        dtdx = dt / p->dx;
        dtdy = dt / p->dy;
        if (index_capa == 0)
            for (i = 1 - mbc; i <= maxm + mbc; i++) { dtdx1d[i + mbc - 1] = dtdx; dtdy1d[i + mbc - 1] = dtdy; }

        for (j = 0; j <= my + 1; j++) {                              /* x-sweeps */
            for (m = 1; m <= meqn; m++)
                for (i = 1 - mbc; i <= mx + mbc; i++) Q1D(q1d, m, i) = A2(qold, meqn, m, i, j);
            if (index_capa > 0)
                for (i = 1 - mbc; i <= mx + mbc; i++) dtdx1d[i + mbc - 1] = dtdx / A2(aux, maux, index_capa, i, j);
            if (maux > 0)
                for (ma = 1; ma <= maux; ma++)
                    for (i = 1 - mbc; i <= mx + mbc; i++) {
                        AUXS(w.aux1, ma, i) = A2(aux, maux, ma, i, j - 1);
                        AUXS(w.aux2, ma, i) = A2(aux, maux, ma, i, j);
                        AUXS(w.aux3, ma, i) = A2(aux, maux, ma, i, j + 1);
                    }
            flux2(1, mx, p, q1d, dtdx1d, w.aux1, w.aux2, w.aux3, p->order, p->transverse,
                  qadd, fadd, gadd, &cfl1d, &w, &ctx);
            cfl = dmax1(cfl, cfl1d);
            if (index_capa == 0) {
                for (m = 1; m <= meqn; m++)
                    for (i = 1; i <= mx; i++) {
                        A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, i)
                            - dtdx * (Q1D(fadd, m, i + 1) - Q1D(fadd, m, i))
                            - dtdy * (GADD(m, 2, i) - GADD(m, 1, i));
                        A2(qnew, meqn, m, i, j - 1) = A2(qnew, meqn, m, i, j - 1) - dtdy * GADD(m, 1, i);
                        A2(qnew, meqn, m, i, j + 1) = A2(qnew, meqn, m, i, j + 1) + dtdy * GADD(m, 2, i);
                    }
            } else {
                for (m = 1; m <= meqn; m++)
                    for (i = 1; i <= mx; i++) {
                        A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, i)
                            - (dtdx * (Q1D(fadd, m, i + 1) - Q1D(fadd, m, i))
                               + dtdy * (GADD(m, 2, i) - GADD(m, 1, i))) / A2(aux, maux, index_capa, i, j);
                        A2(qnew, meqn, m, i, j - 1) = A2(qnew, meqn, m, i, j - 1)
                            - dtdy * GADD(m, 1, i) / A2(aux, maux, index_capa, i, j - 1);
                        A2(qnew, meqn, m, i, j + 1) = A2(qnew, meqn, m, i, j + 1)
                            + dtdy * GADD(m, 2, i) / A2(aux, maux, index_capa, i, j + 1);
                    }
            }
        }

        for (i = 0; i <= mx + 1; i++) {                              /* y-sweeps */
            for (m = 1; m <= meqn; m++)
                for (j = 1 - mbc; j <= my + mbc; j++) Q1D(q1d, m, j) = A2(qold, meqn, m, i, j);
            if (index_capa > 0)
                for (j = 1 - mbc; j <= my + mbc; j++) dtdy1d[j + mbc - 1] = dtdy / A2(aux, maux, index_capa, i, j);
            if (maux > 0)
                for (ma = 1; ma <= maux; ma++)
                    for (j = 1 - mbc; j <= my + mbc; j++) {
                        AUXS(w.aux1, ma, j) = A2(aux, maux, ma, i - 1, j);
                        AUXS(w.aux2, ma, j) = A2(aux, maux, ma, i, j);
                        AUXS(w.aux3, ma, j) = A2(aux, maux, ma, i + 1, j);
                    }
            flux2(2, my, p, q1d, dtdy1d, w.aux1, w.aux2, w.aux3, p->order, p->transverse,
                  qadd, fadd, gadd, &cfl1d, &w, &ctx);
            cfl = dmax1(cfl, cfl1d);
            if (index_capa == 0) {
                for (m = 1; m <= meqn; m++)
                    for (j = 1; j <= my; j++) {
                        A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + (Q1D(qadd, m, j)
                            - dtdy * (Q1D(fadd, m, j + 1) - Q1D(fadd, m, j))
                            - dtdx * (GADD(m, 2, j) - GADD(m, 1, j)));
                        A2(qnew, meqn, m, i - 1, j) = A2(qnew, meqn, m, i - 1, j) - dtdx * GADD(m, 1, j);
                        A2(qnew, meqn, m, i + 1, j) = A2(qnew, meqn, m, i + 1, j) + dtdx * GADD(m, 2, j);
                    }
            } else {
                for (m = 1; m <= meqn; m++)
                    for (j = 1; j <= my; j++) {
                        A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, j)
                            - (dtdy * (Q1D(fadd, m, j + 1) - Q1D(fadd, m, j))
                               + dtdx * (GADD(m, 2, j) - GADD(m, 1, j))) / A2(aux, maux, index_capa, i, j);
                        A2(qnew, meqn, m, i - 1, j) = A2(qnew, meqn, m, i - 1, j)
                            - dtdx * GADD(m, 1, j) / A2(aux, maux, index_capa, i - 1, j);
                        A2(qnew, meqn, m, i + 1, j) = A2(qnew, meqn, m, i + 1, j)
                            + dtdx * GADD(m, 2, j) / A2(aux, maux, index_capa, i + 1, j);
                    }
            }
        }
    }
    *cfl_out = cfl;
    work_free(&w);
    return CLAW2_OK;
}

/* ===================================================================== */
/* step2ds: src/pyclaw/classic/step2ds.f90:55-255 (one sweep per call)     */
/* ===================================================================== */
ORC_API int orc_step2ds(const claw2_problem* p, const double* qold, double* qnew,
                        const double* aux, double dt, int ids, double* cfl_out)
{
    const int meqn = p->num_eqn, mbc = p->num_ghost, mx = p->mx, my = p->my;
    const int maux = p->num_aux, index_capa = p->index_capa + 1;
    orc_work w; orc_ctx ctx;
    double cfl = 0.0, cfl1d, dtdx, dtdy;
    int i, j, m, ma, rc = check_problem(p);
    if (rc) return rc;
    if (ids != 1 && ids != 2) return CLAW2_ERR_INVALID;
    if ((rc = work_alloc(p, &w, &ctx))) { work_free(&w); return rc; }
    {
        double *q1d = w.q1d, *qadd = w.qadd, *fadd = w.fadd;
        double *dtdx1d = w.dtdx1d, *dtdy1d = w.dtdy1d;
        const int maxm = ctx.maxm;
        /* qold may alias qnew (the second sweep passes qbc twice, classic/solver.py:529-531):
         * every slice only writes itself after it has been copied to q1d, so reading
         * through qold here is equivalent. */
        dtdx = dt / p->dx;
        dtdy = dt / p->dy;
        if (index_capa == 0)
            for (i = 1 - mbc; i <= maxm + mbc; i++) { dtdx1d[i + mbc - 1] = dtdx; dtdy1d[i + mbc - 1] = dtdy; }
        if (ids == 1) {
            for (j = 1 - mbc; j <= my + mbc; j++) {
                for (m = 1; m <= meqn; m++)
                    for (i = 1 - mbc; i <= mx + mbc; i++) Q1D(q1d, m, i) = A2(qold, meqn, m, i, j);
                if (index_capa > 0)
                    for (i = 1 - mbc; i <= mx + mbc; i++) dtdx1d[i + mbc - 1] = dtdx / A2(aux, maux, index_capa, i, j);
                if (maux > 0) {
                    for (ma = 1; ma <= maux; ma++)
                        for (i = 1 - mbc; i <= mx + mbc; i++) AUXS(w.aux2, ma, i) = A2(aux, maux, ma, i, j);
                    if (j != 1 - mbc)
                        for (ma = 1; ma <= maux; ma++)
                            for (i = 1 - mbc; i <= mx + mbc; i++) AUXS(w.aux1, ma, i) = A2(aux, maux, ma, i, j - 1);
                    if (j != my + mbc)
                        for (ma = 1; ma <= maux; ma++)
                            for (i = 1 - mbc; i <= mx + mbc; i++) AUXS(w.aux3, ma, i) = A2(aux, maux, ma, i, j + 1);
                }
                flux2(1, mx, p, q1d, dtdx1d, w.aux1, w.aux2, w.aux3, p->order, -1,
                      qadd, fadd, w.gadd, &cfl1d, &w, &ctx);
                cfl = dmax1(cfl, cfl1d);
                for (m = 1; m <= meqn; m++)
                    for (i = 1; i <= mx; i++) {
                        if (index_capa == 0)
                            A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, i)
                                - dtdx * (Q1D(fadd, m, i + 1) - Q1D(fadd, m, i));
                        else
                            A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, i)
                                - dtdx * (Q1D(fadd, m, i + 1) - Q1D(fadd, m, i)) / A2(aux, maux, index_capa, i, j);
                    }
            }
        } else {
            for (i = 1 - mbc; i <= mx + mbc; i++) {
                for (m = 1; m <= meqn; m++)
                    for (j = 1 - mbc; j <= my + mbc; j++) Q1D(q1d, m, j) = A2(qold, meqn, m, i, j);
                if (index_capa > 0)
                    for (j = 1 - mbc; j <= my + mbc; j++) dtdy1d[j + mbc - 1] = dtdy / A2(aux, maux, index_capa, i, j);
                if (maux > 0) {
                    for (ma = 1; ma <= maux; ma++)
                        for (j = 1 - mbc; j <= my + mbc; j++) AUXS(w.aux2, ma, j) = A2(aux, maux, ma, i, j);
                    if (i != 1 - mbc)
                        for (ma = 1; ma <= maux; ma++)
                            for (j = 1 - mbc; j <= my + mbc; j++) AUXS(w.aux1, ma, j) = A2(aux, maux, ma, i - 1, j);
                    if (i != mx + mbc)
                        for (ma = 1; ma <= maux; ma++)
                            for (j = 1 - mbc; j <= my + mbc; j++) AUXS(w.aux3, ma, j) = A2(aux, maux, ma, i + 1, j);
                }
                flux2(2, my, p, q1d, dtdy1d, w.aux1, w.aux2, w.aux3, p->order, -1,
                      qadd, fadd, w.gadd, &cfl1d, &w, &ctx);
                cfl = dmax1(cfl, cfl1d);
                for (m = 1; m <= meqn; m++)
                    for (j = 1; j <= my; j++) {
                        if (index_capa == 0)
                            A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, j)
                                - dtdy * (Q1D(fadd, m, j + 1) - Q1D(fadd, m, j));
                        else
                            A2(qnew, meqn, m, i, j) = A2(qnew, meqn, m, i, j) + Q1D(qadd, m, j)
                                - dtdy * (Q1D(fadd, m, j + 1) - Q1D(fadd, m, j)) / A2(aux, maux, index_capa, i, j);
                    }
            }
        }
    }
    *cfl_out = cfl;
    work_free(&w);
    return CLAW2_OK;
}

/* ===================================================================== */
/* Boundary conditions: src/pyclaw/solver.py:299-434 and :438-576          */
/* ===================================================================== */
/* Fill one side of one dimension of a ghosted Fortran-order array with nc
 * components.  negate = 1-based component to negate for walls (0 = none). */
static void fill_side(const claw2_problem* p, double* a, int nc, int idim, int upper,
                      int bc, int negate)
{
    const int mbc = p->num_ghost, mx = p->mx, my = p->my;
    const int n0 = (idim == 0 ? mx : my) + 2 * mbc;          /* length of the filled axis */
    const int n1 = (idim == 0 ? my : mx) + 2 * mbc;          /* full extent of the other axis */
    int g, o, m;
#define AT(ii, jj) (&a[(size_t)nc * ((idim == 0) ? ((size_t)(ii) + (size_t)(mx + 2 * mbc) * (jj)) \
                                                 : ((size_t)(jj) + (size_t)(mx + 2 * mbc) * (ii)))])
    for (g = 0; g < mbc; g++) {
        int dst, src;
        if (!upper) {
            if (bc == CLAW2_BC_EXTRAP) { dst = g; src = mbc; }
            else if (bc == CLAW2_BC_PERIODIC) { dst = g; src = n0 - 2 * mbc + g; }
            else if (bc == CLAW2_BC_WALL) { dst = g; src = 2 * mbc - 1 - g; }
            else return;
        } else {
            if (bc == CLAW2_BC_EXTRAP) { dst = n0 - 1 - g; src = n0 - mbc - 1; }
            else if (bc == CLAW2_BC_PERIODIC) { dst = n0 - mbc + g; src = mbc + g; }
            else if (bc == CLAW2_BC_WALL) { dst = n0 - 1 - g; src = n0 - 2 * mbc + g; }
            else return;
        }
        for (o = 0; o < n1; o++) {
            double* d = AT(dst, o);
            const double* sp = AT(src, o);
            for (m = 0; m < nc; m++) d[m] = sp[m];
            if (bc == CLAW2_BC_WALL && negate > 0) d[negate - 1] = -sp[negate - 1];
        }
    }
#undef AT
}

ORC_API int orc_fill_ghosts(const claw2_problem* p, double* qbc)
{
    int idim, rc = check_problem(p);
    if (rc) return rc;
    for (idim = 0; idim < 2; idim++) {
        fill_side(p, qbc, p->num_eqn, idim, 0, p->bc_lower[idim], idim + 2);
        fill_side(p, qbc, p->num_eqn, idim, 1, p->bc_upper[idim], idim + 2);
    }
    return CLAW2_OK;
}

ORC_API int orc_fill_aux_ghosts(const claw2_problem* p, double* auxbc)
{
    int idim, rc = check_problem(p);
    if (rc) return rc;
    if (p->num_aux == 0) return CLAW2_OK;
    for (idim = 0; idim < 2; idim++) {
        fill_side(p, auxbc, p->num_aux, idim, 0, p->aux_bc_lower[idim], 0);
        fill_side(p, auxbc, p->num_aux, idim, 1, p->aux_bc_upper[idim], 0);
    }
    return CLAW2_OK;
}

/* One homogeneous step on a ghost-filled qbc, as ClawSolver2D.step_hyperbolic
 * does it (classic/solver.py:513-541): qold = copy, then step2 or the two
 * step2ds sweeps. */
ORC_API int orc_step_hyperbolic(const claw2_problem* p, double* qbc, double* qold_work,
                                const double* auxbc, double dt, double* cfl)
{
    const size_t n = (size_t)p->num_eqn * (p->mx + 2 * p->num_ghost) * (p->my + 2 * p->num_ghost);
    int rc;
    memcpy(qold_work, qbc, n * sizeof(double));
    if (p->transverse >= 0) return orc_step2(p, qold_work, qbc, auxbc, dt, cfl);
    {
        double cx, cy;
        if ((rc = orc_step2ds(p, qold_work, qbc, auxbc, dt, 1, &cx))) return rc;
        if ((rc = orc_step2ds(p, qbc, qbc, auxbc, dt, 2, &cy))) return rc;
        *cfl = cx > cy ? cx : cy;   /* max(cfl_x, cfl_y), classic/solver.py:533 */
    }
    return CLAW2_OK;
}

/* ===================================================================== */
/* evolve_to_time: src/pyclaw/solver.py:582-699                            */
/* ===================================================================== */
/* Host controller init; same contract as claw2_control_init in the product. */
ORC_API int orc_control_init(claw2_control* c, double t, double dt, double tend,
                             double cfl_max, double cfl_desired, double dt_max,
                             int dt_variable, int take_one_step, int64_t max_steps,
                             double prev_cfl)
{
    memset(c, 0, sizeof *c);
    c->t = t; c->dt = dt; c->tstart = t; c->tend = tend;
    c->cfl = prev_cfl;
    c->cfl_max = cfl_max; c->cfl_desired = cfl_desired; c->dt_max = dt_max;
    c->status_cflmax = prev_cfl; c->status_dtmin = dt; c->status_dtmax = dt;
    c->dt_variable = dt_variable; c->take_one_step = take_one_step;
    c->max_steps = max_steps;
    if (!dt_variable) {
        if (take_one_step) c->max_steps = 1;
        else {
            c->max_steps = (int64_t)((tend - t + 1e-10) / dt);
            if (fabs(c->max_steps * dt - (tend - t)) > 1e-5 * (tend - t)) return CLAW2_ERR_INVALID;
        }
    }
    if (dt_variable && cfl_desired > cfl_max) return CLAW2_ERR_INVALID;
    if (tend <= t && !take_one_step) c->max_steps = 0;
    if (c->max_steps <= 0) { c->done = 1; return CLAW2_OK; }
    if (!take_one_step) {                                     /* :637-641 */
        if (c->t + c->dt > c->tend && c->tstart < c->tend) c->dt = c->tend - c->t;
        if (c->tend - c->t - c->dt < 1.e-14 * c->t) c->dt = c->tend - c->t;
    }
    return CLAW2_OK;
}

/* Controller update after a step with CFL number cfl: :650-691 plus the clamp
 * at the top of the next iteration (:637-641).  Returns 1 if accepted. */
ORC_API int orc_control_update(claw2_control* c, double cfl)
{
    int accepted = 0;
    c->cfl = cfl;
    if (cfl <= c->cfl_max) {
        accepted = 1;
        c->status_cflmax = (c->status_cflmax > cfl) ? c->status_cflmax : cfl;   /* max(cfl, cflmax) */
        if (c->dt_variable) c->t += c->dt;
        else c->t = c->tstart + (double)(c->iter + 1) * c->dt;
        c->numsteps++;
    } else {
        c->rejected++;
        if (!c->dt_variable) {
            c->status_cflmax = (cfl > c->status_cflmax) ? cfl : c->status_cflmax;
            c->error = CLAW2_ERR_CFL;
            c->done = 1;
            c->iter++;
            return 0;
        }
    }
    if (c->dt_variable) {
        if (cfl > 0.0) {
            double cand = c->dt * c->cfl_desired / cfl;
            c->dt = (cand < c->dt_max) ? cand : c->dt_max;
            c->status_dtmin = (c->dt < c->status_dtmin) ? c->dt : c->status_dtmin;
            c->status_dtmax = (c->dt > c->status_dtmax) ? c->dt : c->status_dtmax;
        } else {
            c->dt = c->dt_max;
        }
    }
    c->iter++;
    if (c->t >= c->tend || c->take_one_step) { c->done = 1; return accepted; }
    if (c->iter >= c->max_steps) {
        c->done = 1;
        if (c->dt_variable && c->t < c->tend && c->numsteps == c->max_steps) c->error = CLAW2_ERR_MAX_STEPS;
        return accepted;
    }
    if (c->t + c->dt > c->tend && c->tstart < c->tend) c->dt = c->tend - c->t;
    if (c->tend - c->t - c->dt < 1.e-14 * c->t) c->dt = c->tend - c->t;
    return accepted;
}

/* Advance qbc (ghosted, Fortran order; ghosts are refilled every step) until
 * the controller is done.  Non-custom boundary conditions only. */
ORC_API int orc_evolve(const claw2_problem* p, double* qbc, const double* auxbc,
                       claw2_control* c)
{
    const int mbc = p->num_ghost, mx = p->mx, my = p->my, meqn = p->num_eqn;
    const size_t n = (size_t)meqn * (mx + 2 * mbc) * (my + 2 * mbc);
    double *backup, *qold;
    int rc = check_problem(p), idim;
    if (rc) return rc;
    for (idim = 0; idim < 2; idim++)
        if (p->bc_lower[idim] == CLAW2_BC_CUSTOM || p->bc_upper[idim] == CLAW2_BC_CUSTOM) return CLAW2_ERR_UNSUPPORTED;
    backup = malloc(n * sizeof(double));
    qold = malloc(n * sizeof(double));
    if (!backup || !qold) { free(backup); free(qold); return CLAW2_ERR_NOMEM; }
    while (!c->done) {
        double cfl;
        orc_fill_ghosts(p, qbc);
        if (c->dt_variable) memcpy(backup, qbc, n * sizeof(double));
        if ((rc = orc_step_hyperbolic(p, qbc, qold, auxbc, c->dt, &cfl))) break;
        if (!orc_control_update(c, cfl) && c->dt_variable) memcpy(qbc, backup, n * sizeof(double));
    }
    free(backup); free(qold);
    return rc ? rc : c->error;
}

ORC_API int orc_abi_version(void) { return CLAW2_ABI_VERSION; }

/* ===================================================================== */
/* Multi-threaded "gather form" of the same step, for timing the CPU       */
/* baseline on all host cores.  Every slice's flux2 outputs (qadd, fadd,    */
/* gadd) are kept, then each interior cell applies the contributions of     */
/* slices j-1, j, j+1 (then i-1, i, i+1) in the order step2.f90 applies     */
/* them, so the interior is bit-identical to orc_step2 (ghost cells of qnew,*/
/* which the next step's boundary fill overwrites, are not updated).        */
/* The split form parallelises step2ds over its independent slices.        */
/* ===================================================================== */
ORC_API int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static int step2_gather(const claw2_problem* p, const double* qold, double* qnew,
                        const double* aux, double dt, double* cfl_out)
{
    const int meqn = p->num_eqn, mbc = p->num_ghost, mx = p->mx, my = p->my;
    const int maux = p->num_aux, index_capa = p->index_capa + 1;
    const int maxm = mx > my ? mx : my;
    const size_t sl = (size_t)meqn * (maxm + 2 * mbc);        /* one slice of qadd/fadd */
    const int nsx = my + 2, nsy = mx + 2;                        /* slices 0..my+1, 0..mx+1 */
    const int ns = nsx > nsy ? nsx : nsy;
    double *QA = malloc(sl * ns * sizeof(double)), *FA = malloc(sl * ns * sizeof(double));
    double *GA = malloc(2 * sl * ns * sizeof(double)), *CF = malloc(ns * sizeof(double));
    const double dtdx = dt / p->dx, dtdy = dt / p->dy;
    double cfl = 0.0;
    int err = 0, pass;
    if (!QA || !FA || !GA || !CF) { free(QA); free(FA); free(GA); free(CF); return CLAW2_ERR_NOMEM; }

    for (pass = 0; pass < 2; pass++) {
        const int ixy = pass + 1, nslice = pass == 0 ? nsx : nsy, len = pass == 0 ? mx : my;
        int k;
#pragma omp parallel reduction(|:err)
        {
            orc_work w; orc_ctx ctx;
            int s;
            if (work_alloc(p, &w, &ctx)) err |= 1;
            else {
                double *q1d = w.q1d, *dt1 = ixy == 1 ? w.dtdx1d : w.dtdy1d;
                const double dtd = ixy == 1 ? dtdx : dtdy;
                int i, m, ma;
                if (index_capa == 0)
                    for (i = 1 - mbc; i <= maxm + mbc; i++) dt1[i + mbc - 1] = dtd;
#pragma omp for schedule(static)
                for (s = 0; s < nslice; s++) {
                    for (m = 1; m <= meqn; m++)
                        for (i = 1 - mbc; i <= len + mbc; i++)
                            Q1D(q1d, m, i) = ixy == 1 ? A2(qold, meqn, m, i, s) : A2(qold, meqn, m, s, i);
                    if (index_capa > 0)
                        for (i = 1 - mbc; i <= len + mbc; i++)
                            dt1[i + mbc - 1] = dtd / (ixy == 1 ? A2(aux, maux, index_capa, i, s) : A2(aux, maux, index_capa, s, i));
                    if (maux > 0)
                        for (ma = 1; ma <= maux; ma++)
                            for (i = 1 - mbc; i <= len + mbc; i++) {
                                AUXS(w.aux1, ma, i) = ixy == 1 ? A2(aux, maux, ma, i, s - 1) : A2(aux, maux, ma, s - 1, i);
                                AUXS(w.aux2, ma, i) = ixy == 1 ? A2(aux, maux, ma, i, s) : A2(aux, maux, ma, s, i);
                                AUXS(w.aux3, ma, i) = ixy == 1 ? A2(aux, maux, ma, i, s + 1) : A2(aux, maux, ma, s + 1, i);
                            }
                    flux2(ixy, len, p, q1d, dt1, w.aux1, w.aux2, w.aux3, p->order, p->transverse,
                          QA + sl * s, FA + sl * s, GA + 2 * sl * s, &CF[s], &w, &ctx);
                }
            }
            work_free(&w);
        }
        if (err) break;
        for (k = 0; k < nslice; k++) cfl = dmax1(cfl, CF[k]);
        /* gather: interior cells only, contributions in slice order */
#pragma omp parallel for schedule(static)
        for (k = 1; k <= (pass == 0 ? my : mx); k++) {
            int c, m;
            for (m = 1; m <= meqn; m++)
                for (c = 1; c <= len; c++) {
                    const int i = pass == 0 ? c : k, j = pass == 0 ? k : c;
                    const double *qaddS = QA + sl * k, *faddS = FA + sl * k;
                    const double *gm = GA + 2 * sl * (k - 1), *g0 = GA + 2 * sl * k, *gp = GA + 2 * sl * (k + 1);
                    double v = A2(qnew, meqn, m, i, j);
                    const double dtn = pass == 0 ? dtdy : dtdx, dtl = pass == 0 ? dtdx : dtdy;
#define GS(g, mm, kk, ii) (g)[((mm) - 1) + meqn * (((kk) - 1) + 2 * ((ii) + mbc - 1))]
                    if (index_capa == 0) {
                        v = v + dtn * GS(gm, m, 2, c);
                        if (pass == 0)
                            v = v + Q1D(qaddS, m, c) - dtl * (Q1D(faddS, m, c + 1) - Q1D(faddS, m, c))
                                - dtn * (GS(g0, m, 2, c) - GS(g0, m, 1, c));
                        else
                            v = v + (Q1D(qaddS, m, c) - dtl * (Q1D(faddS, m, c + 1) - Q1D(faddS, m, c))
                                     - dtn * (GS(g0, m, 2, c) - GS(g0, m, 1, c)));
                        v = v - dtn * GS(gp, m, 1, c);
                    } else {
                        const double cm = pass == 0 ? A2(aux, maux, index_capa, i, j) : A2(aux, maux, index_capa, i, j);
                        v = v + dtn * GS(gm, m, 2, c) / cm;
                        v = v + Q1D(qaddS, m, c) - (dtl * (Q1D(faddS, m, c + 1) - Q1D(faddS, m, c))
                                                    + dtn * (GS(g0, m, 2, c) - GS(g0, m, 1, c))) / cm;
                        v = v - dtn * GS(gp, m, 1, c) / cm;
                    }
#undef GS
                    A2(qnew, meqn, m, i, j) = v;
                }
        }
    }
    free(QA); free(FA); free(GA); free(CF);
    if (err) return CLAW2_ERR_NOMEM;
    *cfl_out = cfl;
    return CLAW2_OK;
}

static int step2ds_par(const claw2_problem* p, const double* qold, double* qnew,
                       const double* aux, double dt, int ids, double* cfl_out)
{
    const int meqn = p->num_eqn, mbc = p->num_ghost, mx = p->mx, my = p->my;
    const int maux = p->num_aux, index_capa = p->index_capa + 1;
    const int ixy = ids, len = ids == 1 ? mx : my;
    const double dtd = ids == 1 ? dt / p->dx : dt / p->dy;
    double cfl = 0.0;
    int err = 0;
#pragma omp parallel reduction(|:err) reduction(max:cfl)
    {
        orc_work w; orc_ctx ctx;
        int s;
        if (work_alloc(p, &w, &ctx)) err |= 1;
        else {
            double *q1d = w.q1d, *dt1 = ixy == 1 ? w.dtdx1d : w.dtdy1d;
            const int maxm = ctx.maxm;
            int i, m, ma;
            if (index_capa == 0)
                for (i = 1 - mbc; i <= maxm + mbc; i++) dt1[i + mbc - 1] = dtd;
#pragma omp for schedule(static)
            for (s = 1 - mbc; s <= (ids == 1 ? my : mx) + mbc; s++) {
                double cfl1d;
                for (m = 1; m <= meqn; m++)
                    for (i = 1 - mbc; i <= len + mbc; i++)
                        Q1D(q1d, m, i) = ixy == 1 ? A2(qold, meqn, m, i, s) : A2(qold, meqn, m, s, i);
                if (index_capa > 0)
                    for (i = 1 - mbc; i <= len + mbc; i++)
                        dt1[i + mbc - 1] = dtd / (ixy == 1 ? A2(aux, maux, index_capa, i, s) : A2(aux, maux, index_capa, s, i));
                if (maux > 0)
                    for (ma = 1; ma <= maux; ma++)
                        for (i = 1 - mbc; i <= len + mbc; i++)
                            AUXS(w.aux2, ma, i) = ixy == 1 ? A2(aux, maux, ma, i, s) : A2(aux, maux, ma, s, i);
                flux2(ixy, len, p, q1d, dt1, w.aux1, w.aux2, w.aux3, p->order, -1,
                      w.qadd, w.fadd, w.gadd, &cfl1d, &w, &ctx);
                cfl = dmax1(cfl, cfl1d);
                for (m = 1; m <= meqn; m++)
                    for (i = 1; i <= len; i++) {
                        double* d = ixy == 1 ? &A2(qnew, meqn, m, i, s) : &A2(qnew, meqn, m, s, i);
                        double* qadd = w.qadd; double* fadd = w.fadd;
                        if (index_capa == 0)
                            *d = *d + Q1D(qadd, m, i) - dtd * (Q1D(fadd, m, i + 1) - Q1D(fadd, m, i));
                        else
                            *d = *d + Q1D(qadd, m, i) - dtd * (Q1D(fadd, m, i + 1) - Q1D(fadd, m, i))
                                 / (ixy == 1 ? A2(aux, maux, index_capa, i, s) : A2(aux, maux, index_capa, s, i));
                    }
            }
        }
        work_free(&w);
    }
    if (err) return CLAW2_ERR_NOMEM;
    *cfl_out = cfl;
    return CLAW2_OK;
}

ORC_API int orc_step_hyperbolic_omp(const claw2_problem* p, double* qbc, double* qold_work,
                                    const double* auxbc, double dt, double* cfl)
{
    const size_t n = (size_t)p->num_eqn * (p->mx + 2 * p->num_ghost) * (p->my + 2 * p->num_ghost);
    int rc = check_problem(p);
    if (rc) return rc;
    memcpy(qold_work, qbc, n * sizeof(double));
    if (p->transverse >= 0) return step2_gather(p, qold_work, qbc, auxbc, dt, cfl);
    {
        double cx, cy;
        if ((rc = step2ds_par(p, qold_work, qbc, auxbc, dt, 1, &cx))) return rc;
        if ((rc = step2ds_par(p, qbc, qbc, auxbc, dt, 2, &cy))) return rc;
        *cfl = cx > cy ? cx : cy;
    }
    return CLAW2_OK;
}

ORC_API int orc_evolve_omp(const claw2_problem* p, double* qbc, const double* auxbc,
                           claw2_control* c)
{
    const int mbc = p->num_ghost, mx = p->mx, my = p->my, meqn = p->num_eqn;
    const size_t n = (size_t)meqn * (mx + 2 * mbc) * (my + 2 * mbc);
    double *backup, *qold;
    int rc = check_problem(p), idim;
    if (rc) return rc;
    for (idim = 0; idim < 2; idim++)
        if (p->bc_lower[idim] == CLAW2_BC_CUSTOM || p->bc_upper[idim] == CLAW2_BC_CUSTOM) return CLAW2_ERR_UNSUPPORTED;
    backup = malloc(n * sizeof(double));
    qold = malloc(n * sizeof(double));
    if (!backup || !qold) { free(backup); free(qold); return CLAW2_ERR_NOMEM; }
    while (!c->done) {
        double cfl;
        orc_fill_ghosts(p, qbc);
        if (c->dt_variable) memcpy(backup, qbc, n * sizeof(double));
        if ((rc = orc_step_hyperbolic_omp(p, qbc, qold, auxbc, c->dt, &cfl))) break;
        if (!orc_control_update(c, cfl) && c->dt_variable) memcpy(qbc, backup, n * sizeof(double));
    }
    free(backup); free(qold);
    return rc ? rc : c->error;
}
