// hostcheck.cpp — host replay of the device integral arithmetic.
//
// b200jk_hostcheck_cart_quartet evaluates one shell quartet with exactly the
// templates the CUDA kernels run (rys_math.cuh), compiled here as plain C++
// without any device code; b200jk_hostcheck_cart_quartet_fp32 does the same
// in float32 with the float32 tables, as the float32 pass of mixed precision
// does.  They exist to check the kernels' arithmetic against an independent
// CPU integral library without a GPU; the J/K entry points never call them.
#include <math.h>
#include <string.h>
#include <stdint.h>
#include <vector>

#define RYS_TABLE_QUALIFIER static const
#include "rys_math.cuh"
#include "../../include/b200jk.h"

using namespace b200jk;

namespace {

enum { PTR_COORD = 1, ATM_SLOTS = 6 };
enum { ATOM_OF = 0, ANG_OF = 1, NPRIM_OF = 2, NCTR_OF = 3, PTR_EXP = 5, PTR_COEFF = 6, BAS_SLOTS = 8 };

// the padded float64 device layout, built once
const double *padded_table()
{
        alignas(32) static double t[rys_padded_size()];
        static bool done = false;
        if (!done) {
                rys_pad_table(rys_table_data, t);
                done = true;
        }
        return t;
}

template <typename R> const R *table_slice(int nr);
template <> const double *table_slice<double>(int nr) { return padded_table() + rys_padded_offset(nr); }
template <> const float *table_slice<float>(int nr)
{
        alignas(32) static float t[RYS_F_SIZE];
        static bool done = false;
        if (!done) {
                memcpy(t, rys_table_f_data, sizeof(t));
                done = true;
        }
        return t + rys_f_offset(nr);
}

struct HSeg {
        int l, nprim;
        const double *exp, *coef;
        double R[3];
};

// coordinates relative to centre A, differenced in float64, then rounded to
// R: the kernels' convention
template <int LA, int LB, int LC, int LD, typename R>
void host_quartet(const HSeg *s, double *out)
{
        using K = Class4<LA, LB, LC, LD>;
        std::vector<R> G(K::NG, (R)0);
        double Ad[3], Bd[3], Cd[3], Dd[3];
        R A[3], C[3], AB[3], CD[3];
        for (int x = 0; x < 3; x++) {
                Ad[x] = s[0].R[x]; Bd[x] = s[1].R[x]; Cd[x] = s[2].R[x]; Dd[x] = s[3].R[x];
                A[x] = (R)0;
                C[x] = (R)(Cd[x] - Ad[x]);
                AB[x] = (R)(Ad[x] - Bd[x]);
                CD[x] = (R)(Cd[x] - Dd[x]);
        }
        double rab = 0, rcd = 0;
        for (int x = 0; x < 3; x++) {
                rab += (Ad[x] - Bd[x]) * (Ad[x] - Bd[x]);
                rcd += (Cd[x] - Dd[x]) * (Cd[x] - Dd[x]);
        }
        const R *tab = table_slice<R>(K::NR);
        for (int i = 0; i < s[0].nprim; i++)
        for (int j = 0; j < s[1].nprim; j++) {
                const double a = s[0].exp[i], b = s[1].exp[j], p = a + b;
                double P[3];
                for (int x = 0; x < 3; x++) P[x] = (a * Ad[x] + b * Bd[x]) / p;
                const double Kab = s[0].coef[i] * s[1].coef[j] * exp(-a * b / p * rab);
                const R Pr[3] = {(R)(P[0] - Ad[0]), (R)(P[1] - Ad[1]), (R)(P[2] - Ad[2])};
                for (int k = 0; k < s[2].nprim; k++)
                for (int l = 0; l < s[3].nprim; l++) {
                        const double c = s[2].exp[k], d = s[3].exp[l], q = c + d;
                        double Q[3];
                        for (int x = 0; x < 3; x++) Q[x] = (c * Cd[x] + d * Dd[x]) / q;
                        const double Kcd = s[2].coef[k] * s[3].coef[l] * exp(-c * d / q * rcd);
                        const R Qr[3] = {(R)(Q[0] - Ad[0]), (R)(Q[1] - Ad[1]), (R)(Q[2] - Ad[2])};
                        PrimQ<R> sq;
                        prim_setup<R>(sq, (R)p, (R)(0.5 / p), Pr, (R)q, (R)(0.5 / q), Qr, A, C, (R)Kab * (R)Kcd);
                        add_prim_quartet<LA, LB, LC, LD, R>(G.data(), tab, sq, AB, CD);
                }
        }
        for (int t = 0; t < K::NG; t++) out[t] = (double)G[t];
}

template <typename R>
int hostcheck(const int32_t *atm, int natm, const int32_t *bas, int nbas, const double *env, const int32_t *shls,
              double *out)
{
        if (!atm || !bas || !env || !shls || !out) return B200JK_EINVAL;
        HSeg sg[4];
        int ls[4];
        for (int t = 0; t < 4; t++) {
                const int I = shls[t];
                if (I < 0 || I >= nbas) return B200JK_EINVAL;
                const int32_t *b = bas + (size_t)I * BAS_SLOTS;
                if (b[ATOM_OF] < 0 || b[ATOM_OF] >= natm) return B200JK_EINVAL;
                if (b[ANG_OF] < 0 || b[ANG_OF] > 3) return B200JK_EUNSUPPORTED;
                if (b[NCTR_OF] != 1) return B200JK_EUNSUPPORTED;
                sg[t].l = ls[t] = b[ANG_OF];
                sg[t].nprim = b[NPRIM_OF];
                sg[t].exp = env + b[PTR_EXP];
                sg[t].coef = env + b[PTR_COEFF];
                const int pc = atm[(size_t)b[ATOM_OF] * ATM_SLOTS + PTR_COORD];
                for (int x = 0; x < 3; x++) sg[t].R[x] = env[pc + x];
        }
#define B2_HQ(LA, LB, LC, LD) \
        if (ls[0] == LA && ls[1] == LB && ls[2] == LC && ls[3] == LD) { host_quartet<LA, LB, LC, LD, R>(sg, out); return B200JK_OK; }
#define B2_HQ4(LA, LB, LC) B2_HQ(LA, LB, LC, 0) B2_HQ(LA, LB, LC, 1) B2_HQ(LA, LB, LC, 2) B2_HQ(LA, LB, LC, 3)
#define B2_HQ3(LA, LB) B2_HQ4(LA, LB, 0) B2_HQ4(LA, LB, 1) B2_HQ4(LA, LB, 2) B2_HQ4(LA, LB, 3)
        B2_HQ3(0, 0) B2_HQ3(0, 1) B2_HQ3(0, 2) B2_HQ3(0, 3)
        B2_HQ3(1, 0) B2_HQ3(1, 1) B2_HQ3(1, 2) B2_HQ3(1, 3)
        B2_HQ3(2, 0) B2_HQ3(2, 1) B2_HQ3(2, 2) B2_HQ3(2, 3)
        B2_HQ3(3, 0) B2_HQ3(3, 1) B2_HQ3(3, 2) B2_HQ3(3, 3)
#undef B2_HQ3
#undef B2_HQ4
#undef B2_HQ
        return B200JK_EUNSUPPORTED;
}

} // namespace

extern "C" int b200jk_hostcheck_cart_quartet(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                             const double *env, const int32_t *shls, double *out)
{
        return hostcheck<double>(atm, natm, bas, nbas, env, shls, out);
}

extern "C" int b200jk_hostcheck_cart_quartet_fp32(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                                  const double *env, const int32_t *shls, double *out)
{
        return hostcheck<float>(atm, natm, bas, nbas, env, shls, out);
}
