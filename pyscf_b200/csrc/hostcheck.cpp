// hostcheck.cpp — host replay of the device integral arithmetic.
//
// b200jk_hostcheck_cart_quartet evaluates one shell quartet with exactly the
// templates the CUDA kernels run (rys_math.cuh), compiled here as plain C++
// without any device code.  It exists to check the kernels' arithmetic
// against an independent CPU integral library without a GPU; the J/K entry
// points never call it.
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

// the padded device layout, built once
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

struct HSeg {
        int l, nprim;
        const double *exp, *coef;
        double R[3];
};

template <int LA, int LB, int LC, int LD>
void host_quartet(const HSeg *s, double *out)
{
        using K = Class4<LA, LB, LC, LD>;
        std::vector<double> G(K::NG, 0.0);
        double A[3], B[3], C[3], D[3], AB[3], CD[3];
        for (int x = 0; x < 3; x++) {
                A[x] = s[0].R[x]; B[x] = s[1].R[x]; C[x] = s[2].R[x]; D[x] = s[3].R[x];
                AB[x] = A[x] - B[x]; CD[x] = C[x] - D[x];
        }
        const double rab = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
        const double rcd = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
        for (int i = 0; i < s[0].nprim; i++)
        for (int j = 0; j < s[1].nprim; j++) {
                const double a = s[0].exp[i], b = s[1].exp[j], p = a + b;
                const double P[3] = {(a * A[0] + b * B[0]) / p, (a * A[1] + b * B[1]) / p, (a * A[2] + b * B[2]) / p};
                const double Kab = s[0].coef[i] * s[1].coef[j] * exp(-a * b / p * rab);
                for (int k = 0; k < s[2].nprim; k++)
                for (int l = 0; l < s[3].nprim; l++) {
                        const double c = s[2].exp[k], d = s[3].exp[l], q = c + d;
                        const double Q[3] = {(c * C[0] + d * D[0]) / q, (c * C[1] + d * D[1]) / q, (c * C[2] + d * D[2]) / q};
                        const double Kcd = s[2].coef[k] * s[3].coef[l] * exp(-c * d / q * rcd);
                        PrimQ<double> sq;
                        prim_setup(sq, p, 0.5 / p, P, q, 0.5 / q, Q, A, C, Kab * Kcd);
                        add_prim_quartet<LA, LB, LC, LD>(G.data(), padded_table(), sq, AB, CD);
                }
        }
        memcpy(out, G.data(), sizeof(double) * K::NG);
}

} // namespace

extern "C" int b200jk_hostcheck_cart_quartet(const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                             const double *env, const int32_t *shls, double *out)
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
        if (ls[0] == LA && ls[1] == LB && ls[2] == LC && ls[3] == LD) { host_quartet<LA, LB, LC, LD>(sg, out); return B200JK_OK; }
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
