/*
 * hw_mlp_oracle.c -- FP64 CPU restatement of the learned operator's per-point
 * network and loss (TEST INFRASTRUCTURE ONLY: the checker of the GPU training
 * kernels; the network has no counterpart in the reference).
 *
 * Network: 5 -> 32 -> 32 (tanh) -> 4 logits -> softmax.  Parameter layout:
 * W1[32][5], b1[32], W2[32][32], b2[32], W3[4][32], b3[4].  Record: 5 features,
 * G[8][4], T[8]; loss = mean_m ((sum_j w_j G_mj - T_m) / T_m)^2.
 */
#include <math.h>
#include <string.h>

#define NI 5
#define NH 32
#define NK 4
#define NB 8
#define NREC (NI + NK * NB + NB)
#define OW1 0
#define OB1 (OW1 + NH * NI)
#define OW2 (OB1 + NH)
#define OB2 (OW2 + NH * NH)
#define OW3 (OB2 + NH)
#define OB3 (OW3 + NK * NH)
#define NPAR (OB3 + NK)

int or_mlp_nparams(void) { return NPAR; }

/* summed loss over n records; grad (NPAR doubles, summed over records) if non-NULL */
double or_mlp_loss_grad(const double* P, const float* data, int n, double* grad) {
    double L = 0.0;
    if (grad) memset(grad, 0, sizeof(double) * NPAR);
    for (int r = 0; r < n; r++) {
        const float* rec = data + (size_t)r * NREC;
        double x[NI], h1[NH], h2[NH], z[NK], w[NK];
        for (int j = 0; j < NI; j++) x[j] = rec[j];
        for (int i = 0; i < NH; i++) {
            double s = P[OB1 + i];
            for (int j = 0; j < NI; j++) s += P[OW1 + i * NI + j] * x[j];
            h1[i] = tanh(s);
        }
        for (int i = 0; i < NH; i++) {
            double s = P[OB2 + i];
            for (int j = 0; j < NH; j++) s += P[OW2 + i * NH + j] * h1[j];
            h2[i] = tanh(s);
        }
        double zm = -1e300, den = 0.0;
        for (int i = 0; i < NK; i++) {
            double s = P[OB3 + i];
            for (int j = 0; j < NH; j++) s += P[OW3 + i * NH + j] * h2[j];
            z[i] = s;
            if (s > zm) zm = s;
        }
        for (int i = 0; i < NK; i++) { w[i] = exp(z[i] - zm); den += w[i]; }
        for (int i = 0; i < NK; i++) w[i] /= den;
        const float* G = rec + NI;
        const float* T = rec + NI + NK * NB;
        double dw[NK] = {0, 0, 0, 0}, l = 0.0;
        for (int m = 0; m < NB; m++) {
            double p = 0.0;
            for (int j = 0; j < NK; j++) p += w[j] * G[m * NK + j];
            double e = (p - T[m]) / T[m];
            l += e * e;
            double dp = 2.0 * e / ((double)T[m] * NB);
            for (int j = 0; j < NK; j++) dw[j] += dp * G[m * NK + j];
        }
        L += l / NB;
        if (!grad) continue;
        double s = 0.0, dz[NK], d2[NH], d1[NH];
        for (int j = 0; j < NK; j++) s += w[j] * dw[j];
        for (int j = 0; j < NK; j++) dz[j] = w[j] * (dw[j] - s);
        for (int i = 0; i < NH; i++) {
            double a = 0.0;
            for (int k = 0; k < NK; k++) a += P[OW3 + k * NH + i] * dz[k];
            d2[i] = a * (1.0 - h2[i] * h2[i]);
        }
        for (int i = 0; i < NH; i++) {
            double a = 0.0;
            for (int k = 0; k < NH; k++) a += P[OW2 + k * NH + i] * d2[k];
            d1[i] = a * (1.0 - h1[i] * h1[i]);
        }
        for (int i = 0; i < NH; i++) for (int j = 0; j < NI; j++) grad[OW1 + i * NI + j] += d1[i] * x[j];
        for (int i = 0; i < NH; i++) grad[OB1 + i] += d1[i];
        for (int i = 0; i < NH; i++) for (int j = 0; j < NH; j++) grad[OW2 + i * NH + j] += d2[i] * h1[j];
        for (int i = 0; i < NH; i++) grad[OB2 + i] += d2[i];
        for (int i = 0; i < NK; i++) for (int j = 0; j < NH; j++) grad[OW3 + i * NH + j] += dz[i] * h2[j];
        for (int i = 0; i < NK; i++) grad[OB3 + i] += dz[i];
    }
    return L;
}
