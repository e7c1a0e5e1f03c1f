// Generated by janc_b200/csrc/gen_chem.py from 9sp-19r-H2-Air.yaml; do not edit.
// Species: H2, O2, OH, O, H, H2O, HO2, H2O2, N2
#pragma once

#define JB_GEN_NREAC 19
#define JB_GEN_NR 8
#define JB_GEN_NS 9
// structure signature (compared with the loaded mechanism by jb_create)
static const signed char JB_GEN_VF[19][8] = {{1, 1, 0, 0, 0, 0, 0, 0}, {0, 1, 0, 0, 1, 0, 0, 0}, {1, 0, 0, 1, 0, 0, 0, 0}, {1, 0, 1, 0, 0, 0, 0, 0}, {0, 0, 2, 0, 0, 0, 0, 0}, {0, 0, 1, 0, 1, 0, 0, 0}, {0, 0, 0, 0, 2, 0, 0, 0}, {0, 0, 0, 1, 1, 0, 0, 0}, {0, 1, 0, 0, 1, 0, 0, 0}, {0, 0, 0, 0, 1, 0, 1, 0}, {0, 0, 0, 0, 1, 0, 1, 0}, {0, 0, 0, 1, 0, 0, 1, 0}, {0, 0, 1, 0, 0, 0, 1, 0}, {0, 0, 0, 0, 0, 0, 2, 0}, {0, 0, 0, 0, 1, 0, 0, 1}, {0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 1, 0, 0, 0, 0, 1}, {0, 0, 0, 0, 0, 0, 0, 1}, {0, 0, 0, 2, 0, 0, 0, 0}};
static const signed char JB_GEN_VB[19][8] = {{0, 0, 0, 0, 1, 0, 1, 0}, {0, 0, 1, 1, 0, 0, 0, 0}, {0, 0, 1, 0, 1, 0, 0, 0}, {0, 0, 0, 0, 1, 1, 0, 0}, {0, 0, 0, 1, 0, 1, 0, 0}, {0, 0, 0, 0, 0, 1, 0, 0}, {1, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 1, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 1, 0}, {0, 0, 2, 0, 0, 0, 0, 0}, {0, 0, 0, 1, 0, 1, 0, 0}, {0, 1, 1, 0, 0, 0, 0, 0}, {0, 1, 0, 0, 0, 1, 0, 0}, {0, 1, 0, 0, 0, 0, 0, 1}, {1, 0, 0, 0, 0, 0, 1, 0}, {0, 0, 1, 0, 0, 0, 1, 0}, {0, 0, 0, 0, 0, 1, 1, 0}, {0, 0, 2, 0, 0, 0, 0, 0}, {0, 1, 0, 0, 0, 0, 0, 0}};
static const signed char JB_GEN_TBNZ[19][9] = {{0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {1, 1, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1, 1}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 0}, {1, 1, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1, 1}};
static const signed char JB_GEN_ISTB[19] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1};
static const signed char JB_GEN_VSUM[19] = {0, 0, 0, 0, 0, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1};

#ifdef JB_NS
namespace jb {
namespace JB_NS {
namespace {

// Phase A: rates of every reaction for one cell.  Writes q_i = kf - kb,
// F_i = M_i kf and B_i = M_i kb to shared memory (layout [i][3][stride])
// and accumulates w_k = sum_i dv_ik M_i q_i.  Xc: clipped concentrations;
// E, iE: exp(g_k) and 1 / exp(g_k); Tp = T / pref, pT = pref / T.
__device__ __forceinline__ void chem_rates_gen(const MP& m, double lT, double invT, double Tp, double pT,
    const double* X, const double* Xc, const double* E, const double* iE, double* sh, int stride,
    double* wk) {
  wk[0] = 0.0;
  wk[1] = 0.0;
  wk[2] = 0.0;
  wk[3] = 0.0;
  wk[4] = 0.0;
  wk[5] = 0.0;
  wk[6] = 0.0;
  wk[7] = 0.0;
  {  // reaction 0
    const double k0 = exp(m.lnA[0] + m.B[0] * lT - m.EaR[0] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[0] * Xc[1];
    const double kb = k0 * E[0] * E[1] * iE[4] * iE[6] * Xc[4] * Xc[6];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[0] -= Mq;
    wk[1] -= Mq;
    wk[4] += Mq;
    wk[6] += Mq;
    sh[(0 + 0) * stride] = q;
    sh[(0 + 1) * stride] = Mi * kf;
    sh[(0 + 2) * stride] = Mi * kb;
  }
  {  // reaction 1
    const double k0 = exp(m.lnA[1] + m.B[1] * lT - m.EaR[1] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[1] * Xc[4];
    const double kb = k0 * E[1] * E[4] * iE[2] * iE[3] * Xc[2] * Xc[3];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[1] -= Mq;
    wk[2] += Mq;
    wk[3] += Mq;
    wk[4] -= Mq;
    sh[(3 + 0) * stride] = q;
    sh[(3 + 1) * stride] = Mi * kf;
    sh[(3 + 2) * stride] = Mi * kb;
  }
  {  // reaction 2
    const double k0 = exp(m.lnA[2] + m.B[2] * lT - m.EaR[2] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[0] * Xc[3];
    const double kb = k0 * E[0] * E[3] * iE[2] * iE[4] * Xc[2] * Xc[4];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[0] -= Mq;
    wk[2] += Mq;
    wk[3] -= Mq;
    wk[4] += Mq;
    sh[(6 + 0) * stride] = q;
    sh[(6 + 1) * stride] = Mi * kf;
    sh[(6 + 2) * stride] = Mi * kb;
  }
  {  // reaction 3
    const double k0 = exp(m.lnA[3] + m.B[3] * lT - m.EaR[3] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[0] * Xc[2];
    const double kb = k0 * E[0] * E[2] * iE[4] * iE[5] * Xc[4] * Xc[5];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[0] -= Mq;
    wk[2] -= Mq;
    wk[4] += Mq;
    wk[5] += Mq;
    sh[(9 + 0) * stride] = q;
    sh[(9 + 1) * stride] = Mi * kf;
    sh[(9 + 2) * stride] = Mi * kb;
  }
  {  // reaction 4
    const double k0 = exp(m.lnA[4] + m.B[4] * lT - m.EaR[4] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[2] * Xc[2];
    const double kb = k0 * E[2] * E[2] * iE[3] * iE[5] * Xc[3] * Xc[5];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] += -2.0 * Mq;
    wk[3] += Mq;
    wk[5] += Mq;
    sh[(12 + 0) * stride] = q;
    sh[(12 + 1) * stride] = Mi * kf;
    sh[(12 + 2) * stride] = Mi * kb;
  }
  {  // reaction 5
    const double k0 = exp(m.lnA[5] + m.B[5] * lT - m.EaR[5] * invT);
    const double Mi = m.tb[5][0] * X[0] + m.tb[5][1] * X[1] + m.tb[5][2] * X[2] + m.tb[5][3] * X[3] + m.tb[5][4] * X[4] + m.tb[5][5] * X[5] + m.tb[5][6] * X[6] + m.tb[5][7] * X[7] + m.tb[5][8] * X[8];
    const double kf = k0 * Xc[2] * Xc[4];
    const double kb = k0 * E[2] * E[4] * iE[5] * pT * Xc[5];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] -= Mq;
    wk[4] -= Mq;
    wk[5] += Mq;
    sh[(15 + 0) * stride] = q;
    sh[(15 + 1) * stride] = Mi * kf;
    sh[(15 + 2) * stride] = Mi * kb;
  }
  {  // reaction 6
    const double k0 = exp(m.lnA[6] + m.B[6] * lT - m.EaR[6] * invT);
    const double Mi = m.tb[6][0] * X[0] + m.tb[6][1] * X[1] + m.tb[6][2] * X[2] + m.tb[6][3] * X[3] + m.tb[6][4] * X[4] + m.tb[6][5] * X[5] + m.tb[6][6] * X[6] + m.tb[6][7] * X[7] + m.tb[6][8] * X[8];
    const double kf = k0 * Xc[4] * Xc[4];
    const double kb = k0 * E[4] * E[4] * iE[0] * pT * Xc[0];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[0] += Mq;
    wk[4] += -2.0 * Mq;
    sh[(18 + 0) * stride] = q;
    sh[(18 + 1) * stride] = Mi * kf;
    sh[(18 + 2) * stride] = Mi * kb;
  }
  {  // reaction 7
    const double k0 = exp(m.lnA[7] + m.B[7] * lT - m.EaR[7] * invT);
    const double Mi = m.tb[7][0] * X[0] + m.tb[7][1] * X[1] + m.tb[7][2] * X[2] + m.tb[7][3] * X[3] + m.tb[7][4] * X[4] + m.tb[7][5] * X[5] + m.tb[7][6] * X[6] + m.tb[7][7] * X[7] + m.tb[7][8] * X[8];
    const double kf = k0 * Xc[3] * Xc[4];
    const double kb = k0 * E[3] * E[4] * iE[2] * pT * Xc[2];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] += Mq;
    wk[3] -= Mq;
    wk[4] -= Mq;
    sh[(21 + 0) * stride] = q;
    sh[(21 + 1) * stride] = Mi * kf;
    sh[(21 + 2) * stride] = Mi * kb;
  }
  {  // reaction 8
    const double k0 = exp(m.lnA[8] + m.B[8] * lT - m.EaR[8] * invT);
    const double Mi = m.tb[8][0] * X[0] + m.tb[8][1] * X[1] + m.tb[8][2] * X[2] + m.tb[8][3] * X[3] + m.tb[8][4] * X[4] + m.tb[8][5] * X[5] + m.tb[8][6] * X[6] + m.tb[8][7] * X[7] + m.tb[8][8] * X[8];
    const double kf = k0 * Xc[1] * Xc[4];
    const double kb = k0 * E[1] * E[4] * iE[6] * pT * Xc[6];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[1] -= Mq;
    wk[4] -= Mq;
    wk[6] += Mq;
    sh[(24 + 0) * stride] = q;
    sh[(24 + 1) * stride] = Mi * kf;
    sh[(24 + 2) * stride] = Mi * kb;
  }
  {  // reaction 9
    const double k0 = exp(m.lnA[9] + m.B[9] * lT - m.EaR[9] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[4] * Xc[6];
    const double kb = k0 * E[4] * E[6] * iE[2] * iE[2] * Xc[2] * Xc[2];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] += 2.0 * Mq;
    wk[4] -= Mq;
    wk[6] -= Mq;
    sh[(27 + 0) * stride] = q;
    sh[(27 + 1) * stride] = Mi * kf;
    sh[(27 + 2) * stride] = Mi * kb;
  }
  {  // reaction 10
    const double k0 = exp(m.lnA[10] + m.B[10] * lT - m.EaR[10] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[4] * Xc[6];
    const double kb = k0 * E[4] * E[6] * iE[3] * iE[5] * Xc[3] * Xc[5];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[3] += Mq;
    wk[4] -= Mq;
    wk[5] += Mq;
    wk[6] -= Mq;
    sh[(30 + 0) * stride] = q;
    sh[(30 + 1) * stride] = Mi * kf;
    sh[(30 + 2) * stride] = Mi * kb;
  }
  {  // reaction 11
    const double k0 = exp(m.lnA[11] + m.B[11] * lT - m.EaR[11] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[3] * Xc[6];
    const double kb = k0 * E[3] * E[6] * iE[1] * iE[2] * Xc[1] * Xc[2];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[1] += Mq;
    wk[2] += Mq;
    wk[3] -= Mq;
    wk[6] -= Mq;
    sh[(33 + 0) * stride] = q;
    sh[(33 + 1) * stride] = Mi * kf;
    sh[(33 + 2) * stride] = Mi * kb;
  }
  {  // reaction 12
    const double k0 = exp(m.lnA[12] + m.B[12] * lT - m.EaR[12] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[2] * Xc[6];
    const double kb = k0 * E[2] * E[6] * iE[1] * iE[5] * Xc[1] * Xc[5];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[1] += Mq;
    wk[2] -= Mq;
    wk[5] += Mq;
    wk[6] -= Mq;
    sh[(36 + 0) * stride] = q;
    sh[(36 + 1) * stride] = Mi * kf;
    sh[(36 + 2) * stride] = Mi * kb;
  }
  {  // reaction 13
    const double k0 = exp(m.lnA[13] + m.B[13] * lT - m.EaR[13] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[6] * Xc[6];
    const double kb = k0 * E[6] * E[6] * iE[1] * iE[7] * Xc[1] * Xc[7];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[1] += Mq;
    wk[6] += -2.0 * Mq;
    wk[7] += Mq;
    sh[(39 + 0) * stride] = q;
    sh[(39 + 1) * stride] = Mi * kf;
    sh[(39 + 2) * stride] = Mi * kb;
  }
  {  // reaction 14
    const double k0 = exp(m.lnA[14] + m.B[14] * lT - m.EaR[14] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[4] * Xc[7];
    const double kb = k0 * E[4] * E[7] * iE[0] * iE[6] * Xc[0] * Xc[6];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[0] += Mq;
    wk[4] -= Mq;
    wk[6] += Mq;
    wk[7] -= Mq;
    sh[(42 + 0) * stride] = q;
    sh[(42 + 1) * stride] = Mi * kf;
    sh[(42 + 2) * stride] = Mi * kb;
  }
  {  // reaction 15
    const double k0 = exp(m.lnA[15] + m.B[15] * lT - m.EaR[15] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[3] * Xc[7];
    const double kb = k0 * E[3] * E[7] * iE[2] * iE[6] * Xc[2] * Xc[6];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] += Mq;
    wk[3] -= Mq;
    wk[6] += Mq;
    wk[7] -= Mq;
    sh[(45 + 0) * stride] = q;
    sh[(45 + 1) * stride] = Mi * kf;
    sh[(45 + 2) * stride] = Mi * kb;
  }
  {  // reaction 16
    const double k0 = exp(m.lnA[16] + m.B[16] * lT - m.EaR[16] * invT);
    const double Mi = 1.0;
    const double kf = k0 * Xc[2] * Xc[7];
    const double kb = k0 * E[2] * E[7] * iE[5] * iE[6] * Xc[5] * Xc[6];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] -= Mq;
    wk[5] += Mq;
    wk[6] += Mq;
    wk[7] -= Mq;
    sh[(48 + 0) * stride] = q;
    sh[(48 + 1) * stride] = Mi * kf;
    sh[(48 + 2) * stride] = Mi * kb;
  }
  {  // reaction 17
    const double k0 = exp(m.lnA[17] + m.B[17] * lT - m.EaR[17] * invT);
    const double Mi = m.tb[17][0] * X[0] + m.tb[17][1] * X[1] + m.tb[17][2] * X[2] + m.tb[17][3] * X[3] + m.tb[17][4] * X[4] + m.tb[17][5] * X[5] + m.tb[17][6] * X[6] + m.tb[17][7] * X[7] + m.tb[17][8] * X[8];
    const double kf = k0 * Xc[7];
    const double kb = k0 * E[7] * iE[2] * iE[2] * Tp * Xc[2] * Xc[2];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[2] += 2.0 * Mq;
    wk[7] -= Mq;
    sh[(51 + 0) * stride] = q;
    sh[(51 + 1) * stride] = Mi * kf;
    sh[(51 + 2) * stride] = Mi * kb;
  }
  {  // reaction 18
    const double k0 = exp(m.lnA[18] + m.B[18] * lT - m.EaR[18] * invT);
    const double Mi = m.tb[18][0] * X[0] + m.tb[18][1] * X[1] + m.tb[18][2] * X[2] + m.tb[18][3] * X[3] + m.tb[18][4] * X[4] + m.tb[18][5] * X[5] + m.tb[18][6] * X[6] + m.tb[18][7] * X[7] + m.tb[18][8] * X[8];
    const double kf = k0 * Xc[3] * Xc[3];
    const double kb = k0 * E[3] * E[3] * iE[1] * pT * Xc[1];
    const double q = kf - kb;
    const double Mq = Mi * q;
    wk[1] += Mq;
    wk[3] += -2.0 * Mq;
    sh[(54 + 0) * stride] = q;
    sh[(54 + 1) * stride] = Mi * kf;
    sh[(54 + 2) * stride] = Mi * kb;
  }
}

// Phase B: the analytic Jacobian J[k][n] (without the M_k row factor).
__device__ __forceinline__ void chem_jac_gen(const MP& m, const double* rMX, const double* sh,
    int stride, double (&J)[8][8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int n = 0; n < 8; ++n) J[k][n] = 0.0;
  {  // reaction 0
    const double F = sh[(0 + 1) * stride];
    const double B = sh[(0 + 2) * stride];
    { const double c = (F) * rMX[0];
      J[0][0] -= c;
      J[1][0] -= c;
      J[4][0] += c;
      J[6][0] += c;
    }
    { const double c = (F) * rMX[1];
      J[0][1] -= c;
      J[1][1] -= c;
      J[4][1] += c;
      J[6][1] += c;
    }
    { const double c = (-B) * rMX[4];
      J[0][4] -= c;
      J[1][4] -= c;
      J[4][4] += c;
      J[6][4] += c;
    }
    { const double c = (-B) * rMX[6];
      J[0][6] -= c;
      J[1][6] -= c;
      J[4][6] += c;
      J[6][6] += c;
    }
  }
  {  // reaction 1
    const double F = sh[(3 + 1) * stride];
    const double B = sh[(3 + 2) * stride];
    { const double c = (F) * rMX[1];
      J[1][1] -= c;
      J[2][1] += c;
      J[3][1] += c;
      J[4][1] -= c;
    }
    { const double c = (-B) * rMX[2];
      J[1][2] -= c;
      J[2][2] += c;
      J[3][2] += c;
      J[4][2] -= c;
    }
    { const double c = (-B) * rMX[3];
      J[1][3] -= c;
      J[2][3] += c;
      J[3][3] += c;
      J[4][3] -= c;
    }
    { const double c = (F) * rMX[4];
      J[1][4] -= c;
      J[2][4] += c;
      J[3][4] += c;
      J[4][4] -= c;
    }
  }
  {  // reaction 2
    const double F = sh[(6 + 1) * stride];
    const double B = sh[(6 + 2) * stride];
    { const double c = (F) * rMX[0];
      J[0][0] -= c;
      J[2][0] += c;
      J[3][0] -= c;
      J[4][0] += c;
    }
    { const double c = (-B) * rMX[2];
      J[0][2] -= c;
      J[2][2] += c;
      J[3][2] -= c;
      J[4][2] += c;
    }
    { const double c = (F) * rMX[3];
      J[0][3] -= c;
      J[2][3] += c;
      J[3][3] -= c;
      J[4][3] += c;
    }
    { const double c = (-B) * rMX[4];
      J[0][4] -= c;
      J[2][4] += c;
      J[3][4] -= c;
      J[4][4] += c;
    }
  }
  {  // reaction 3
    const double F = sh[(9 + 1) * stride];
    const double B = sh[(9 + 2) * stride];
    { const double c = (F) * rMX[0];
      J[0][0] -= c;
      J[2][0] -= c;
      J[4][0] += c;
      J[5][0] += c;
    }
    { const double c = (F) * rMX[2];
      J[0][2] -= c;
      J[2][2] -= c;
      J[4][2] += c;
      J[5][2] += c;
    }
    { const double c = (-B) * rMX[4];
      J[0][4] -= c;
      J[2][4] -= c;
      J[4][4] += c;
      J[5][4] += c;
    }
    { const double c = (-B) * rMX[5];
      J[0][5] -= c;
      J[2][5] -= c;
      J[4][5] += c;
      J[5][5] += c;
    }
  }
  {  // reaction 4
    const double F = sh[(12 + 1) * stride];
    const double B = sh[(12 + 2) * stride];
    { const double c = (2.0 * F) * rMX[2];
      J[2][2] += -2.0 * c;
      J[3][2] += c;
      J[5][2] += c;
    }
    { const double c = (-B) * rMX[3];
      J[2][3] += -2.0 * c;
      J[3][3] += c;
      J[5][3] += c;
    }
    { const double c = (-B) * rMX[5];
      J[2][5] += -2.0 * c;
      J[3][5] += c;
      J[5][5] += c;
    }
  }
  {  // reaction 5
    const double q = sh[(15 + 0) * stride];
    const double F = sh[(15 + 1) * stride];
    const double B = sh[(15 + 2) * stride];
    { const double c = q * m.tbinvM[5][0];
      J[2][0] -= c;
      J[4][0] -= c;
      J[5][0] += c;
    }
    { const double c = q * m.tbinvM[5][1];
      J[2][1] -= c;
      J[4][1] -= c;
      J[5][1] += c;
    }
    { const double c = q * m.tbinvM[5][2] + (F) * rMX[2];
      J[2][2] -= c;
      J[4][2] -= c;
      J[5][2] += c;
    }
    { const double c = q * m.tbinvM[5][3];
      J[2][3] -= c;
      J[4][3] -= c;
      J[5][3] += c;
    }
    { const double c = q * m.tbinvM[5][4] + (F) * rMX[4];
      J[2][4] -= c;
      J[4][4] -= c;
      J[5][4] += c;
    }
    { const double c = q * m.tbinvM[5][5] + (-B) * rMX[5];
      J[2][5] -= c;
      J[4][5] -= c;
      J[5][5] += c;
    }
    { const double c = q * m.tbinvM[5][6];
      J[2][6] -= c;
      J[4][6] -= c;
      J[5][6] += c;
    }
    { const double c = q * m.tbinvM[5][7];
      J[2][7] -= c;
      J[4][7] -= c;
      J[5][7] += c;
    }
  }
  {  // reaction 6
    const double q = sh[(18 + 0) * stride];
    const double F = sh[(18 + 1) * stride];
    const double B = sh[(18 + 2) * stride];
    { const double c = q * m.tbinvM[6][0] + (-B) * rMX[0];
      J[0][0] += c;
      J[4][0] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][1];
      J[0][1] += c;
      J[4][1] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][2];
      J[0][2] += c;
      J[4][2] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][3];
      J[0][3] += c;
      J[4][3] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][4] + (2.0 * F) * rMX[4];
      J[0][4] += c;
      J[4][4] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][5];
      J[0][5] += c;
      J[4][5] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][6];
      J[0][6] += c;
      J[4][6] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[6][7];
      J[0][7] += c;
      J[4][7] += -2.0 * c;
    }
  }
  {  // reaction 7
    const double q = sh[(21 + 0) * stride];
    const double F = sh[(21 + 1) * stride];
    const double B = sh[(21 + 2) * stride];
    { const double c = q * m.tbinvM[7][0];
      J[2][0] += c;
      J[3][0] -= c;
      J[4][0] -= c;
    }
    { const double c = q * m.tbinvM[7][1];
      J[2][1] += c;
      J[3][1] -= c;
      J[4][1] -= c;
    }
    { const double c = q * m.tbinvM[7][2] + (-B) * rMX[2];
      J[2][2] += c;
      J[3][2] -= c;
      J[4][2] -= c;
    }
    { const double c = q * m.tbinvM[7][3] + (F) * rMX[3];
      J[2][3] += c;
      J[3][3] -= c;
      J[4][3] -= c;
    }
    { const double c = q * m.tbinvM[7][4] + (F) * rMX[4];
      J[2][4] += c;
      J[3][4] -= c;
      J[4][4] -= c;
    }
    { const double c = q * m.tbinvM[7][5];
      J[2][5] += c;
      J[3][5] -= c;
      J[4][5] -= c;
    }
    { const double c = q * m.tbinvM[7][6];
      J[2][6] += c;
      J[3][6] -= c;
      J[4][6] -= c;
    }
    { const double c = q * m.tbinvM[7][7];
      J[2][7] += c;
      J[3][7] -= c;
      J[4][7] -= c;
    }
  }
  {  // reaction 8
    const double q = sh[(24 + 0) * stride];
    const double F = sh[(24 + 1) * stride];
    const double B = sh[(24 + 2) * stride];
    { const double c = q * m.tbinvM[8][0];
      J[1][0] -= c;
      J[4][0] -= c;
      J[6][0] += c;
    }
    { const double c = q * m.tbinvM[8][1] + (F) * rMX[1];
      J[1][1] -= c;
      J[4][1] -= c;
      J[6][1] += c;
    }
    { const double c = q * m.tbinvM[8][2];
      J[1][2] -= c;
      J[4][2] -= c;
      J[6][2] += c;
    }
    { const double c = q * m.tbinvM[8][3];
      J[1][3] -= c;
      J[4][3] -= c;
      J[6][3] += c;
    }
    { const double c = q * m.tbinvM[8][4] + (F) * rMX[4];
      J[1][4] -= c;
      J[4][4] -= c;
      J[6][4] += c;
    }
    { const double c = q * m.tbinvM[8][5];
      J[1][5] -= c;
      J[4][5] -= c;
      J[6][5] += c;
    }
    { const double c = q * m.tbinvM[8][6] + (-B) * rMX[6];
      J[1][6] -= c;
      J[4][6] -= c;
      J[6][6] += c;
    }
    { const double c = q * m.tbinvM[8][7];
      J[1][7] -= c;
      J[4][7] -= c;
      J[6][7] += c;
    }
  }
  {  // reaction 9
    const double F = sh[(27 + 1) * stride];
    const double B = sh[(27 + 2) * stride];
    { const double c = (-2.0 * B) * rMX[2];
      J[2][2] += 2.0 * c;
      J[4][2] -= c;
      J[6][2] -= c;
    }
    { const double c = (F) * rMX[4];
      J[2][4] += 2.0 * c;
      J[4][4] -= c;
      J[6][4] -= c;
    }
    { const double c = (F) * rMX[6];
      J[2][6] += 2.0 * c;
      J[4][6] -= c;
      J[6][6] -= c;
    }
  }
  {  // reaction 10
    const double F = sh[(30 + 1) * stride];
    const double B = sh[(30 + 2) * stride];
    { const double c = (-B) * rMX[3];
      J[3][3] += c;
      J[4][3] -= c;
      J[5][3] += c;
      J[6][3] -= c;
    }
    { const double c = (F) * rMX[4];
      J[3][4] += c;
      J[4][4] -= c;
      J[5][4] += c;
      J[6][4] -= c;
    }
    { const double c = (-B) * rMX[5];
      J[3][5] += c;
      J[4][5] -= c;
      J[5][5] += c;
      J[6][5] -= c;
    }
    { const double c = (F) * rMX[6];
      J[3][6] += c;
      J[4][6] -= c;
      J[5][6] += c;
      J[6][6] -= c;
    }
  }
  {  // reaction 11
    const double F = sh[(33 + 1) * stride];
    const double B = sh[(33 + 2) * stride];
    { const double c = (-B) * rMX[1];
      J[1][1] += c;
      J[2][1] += c;
      J[3][1] -= c;
      J[6][1] -= c;
    }
    { const double c = (-B) * rMX[2];
      J[1][2] += c;
      J[2][2] += c;
      J[3][2] -= c;
      J[6][2] -= c;
    }
    { const double c = (F) * rMX[3];
      J[1][3] += c;
      J[2][3] += c;
      J[3][3] -= c;
      J[6][3] -= c;
    }
    { const double c = (F) * rMX[6];
      J[1][6] += c;
      J[2][6] += c;
      J[3][6] -= c;
      J[6][6] -= c;
    }
  }
  {  // reaction 12
    const double F = sh[(36 + 1) * stride];
    const double B = sh[(36 + 2) * stride];
    { const double c = (-B) * rMX[1];
      J[1][1] += c;
      J[2][1] -= c;
      J[5][1] += c;
      J[6][1] -= c;
    }
    { const double c = (F) * rMX[2];
      J[1][2] += c;
      J[2][2] -= c;
      J[5][2] += c;
      J[6][2] -= c;
    }
    { const double c = (-B) * rMX[5];
      J[1][5] += c;
      J[2][5] -= c;
      J[5][5] += c;
      J[6][5] -= c;
    }
    { const double c = (F) * rMX[6];
      J[1][6] += c;
      J[2][6] -= c;
      J[5][6] += c;
      J[6][6] -= c;
    }
  }
  {  // reaction 13
    const double F = sh[(39 + 1) * stride];
    const double B = sh[(39 + 2) * stride];
    { const double c = (-B) * rMX[1];
      J[1][1] += c;
      J[6][1] += -2.0 * c;
      J[7][1] += c;
    }
    { const double c = (2.0 * F) * rMX[6];
      J[1][6] += c;
      J[6][6] += -2.0 * c;
      J[7][6] += c;
    }
    { const double c = (-B) * rMX[7];
      J[1][7] += c;
      J[6][7] += -2.0 * c;
      J[7][7] += c;
    }
  }
  {  // reaction 14
    const double F = sh[(42 + 1) * stride];
    const double B = sh[(42 + 2) * stride];
    { const double c = (-B) * rMX[0];
      J[0][0] += c;
      J[4][0] -= c;
      J[6][0] += c;
      J[7][0] -= c;
    }
    { const double c = (F) * rMX[4];
      J[0][4] += c;
      J[4][4] -= c;
      J[6][4] += c;
      J[7][4] -= c;
    }
    { const double c = (-B) * rMX[6];
      J[0][6] += c;
      J[4][6] -= c;
      J[6][6] += c;
      J[7][6] -= c;
    }
    { const double c = (F) * rMX[7];
      J[0][7] += c;
      J[4][7] -= c;
      J[6][7] += c;
      J[7][7] -= c;
    }
  }
  {  // reaction 15
    const double F = sh[(45 + 1) * stride];
    const double B = sh[(45 + 2) * stride];
    { const double c = (-B) * rMX[2];
      J[2][2] += c;
      J[3][2] -= c;
      J[6][2] += c;
      J[7][2] -= c;
    }
    { const double c = (F) * rMX[3];
      J[2][3] += c;
      J[3][3] -= c;
      J[6][3] += c;
      J[7][3] -= c;
    }
    { const double c = (-B) * rMX[6];
      J[2][6] += c;
      J[3][6] -= c;
      J[6][6] += c;
      J[7][6] -= c;
    }
    { const double c = (F) * rMX[7];
      J[2][7] += c;
      J[3][7] -= c;
      J[6][7] += c;
      J[7][7] -= c;
    }
  }
  {  // reaction 16
    const double F = sh[(48 + 1) * stride];
    const double B = sh[(48 + 2) * stride];
    { const double c = (F) * rMX[2];
      J[2][2] -= c;
      J[5][2] += c;
      J[6][2] += c;
      J[7][2] -= c;
    }
    { const double c = (-B) * rMX[5];
      J[2][5] -= c;
      J[5][5] += c;
      J[6][5] += c;
      J[7][5] -= c;
    }
    { const double c = (-B) * rMX[6];
      J[2][6] -= c;
      J[5][6] += c;
      J[6][6] += c;
      J[7][6] -= c;
    }
    { const double c = (F) * rMX[7];
      J[2][7] -= c;
      J[5][7] += c;
      J[6][7] += c;
      J[7][7] -= c;
    }
  }
  {  // reaction 17
    const double q = sh[(51 + 0) * stride];
    const double F = sh[(51 + 1) * stride];
    const double B = sh[(51 + 2) * stride];
    { const double c = q * m.tbinvM[17][0];
      J[2][0] += 2.0 * c;
      J[7][0] -= c;
    }
    { const double c = q * m.tbinvM[17][1];
      J[2][1] += 2.0 * c;
      J[7][1] -= c;
    }
    { const double c = q * m.tbinvM[17][2] + (-2.0 * B) * rMX[2];
      J[2][2] += 2.0 * c;
      J[7][2] -= c;
    }
    { const double c = q * m.tbinvM[17][3];
      J[2][3] += 2.0 * c;
      J[7][3] -= c;
    }
    { const double c = q * m.tbinvM[17][4];
      J[2][4] += 2.0 * c;
      J[7][4] -= c;
    }
    { const double c = q * m.tbinvM[17][5];
      J[2][5] += 2.0 * c;
      J[7][5] -= c;
    }
    { const double c = q * m.tbinvM[17][6];
      J[2][6] += 2.0 * c;
      J[7][6] -= c;
    }
    { const double c = q * m.tbinvM[17][7] + (F) * rMX[7];
      J[2][7] += 2.0 * c;
      J[7][7] -= c;
    }
  }
  {  // reaction 18
    const double q = sh[(54 + 0) * stride];
    const double F = sh[(54 + 1) * stride];
    const double B = sh[(54 + 2) * stride];
    { const double c = q * m.tbinvM[18][0];
      J[1][0] += c;
      J[3][0] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][1] + (-B) * rMX[1];
      J[1][1] += c;
      J[3][1] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][2];
      J[1][2] += c;
      J[3][2] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][3] + (2.0 * F) * rMX[3];
      J[1][3] += c;
      J[3][3] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][4];
      J[1][4] += c;
      J[3][4] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][5];
      J[1][5] += c;
      J[3][5] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][6];
      J[1][6] += c;
      J[3][6] += -2.0 * c;
    }
    { const double c = q * m.tbinvM[18][7];
      J[1][7] += c;
      J[3][7] += -2.0 * c;
    }
  }
}

}  // namespace
}  // namespace JB_NS
}  // namespace jb
#endif
