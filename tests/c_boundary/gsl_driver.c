/*
 * A C caller of the engine written the way the reference drives its RHS: the RHS
 * registered in a gsl_odeiv_system-shaped struct (1d/functions.c:71-89) and the
 * evolve loop of ode_solver_Ham (1d/functions.c:546-553),
 *
 *     for each output time ti:  while (t < ti) status = evolve_apply(..., &t, ti, &h, y);
 *
 * with hw_evolve_apply in place of gsl_odeiv_evolve_apply and hw_gsl_rhs in place
 * of rhs_HsF1/2/3.  Compiled against include/hawassi_b200.h only.
 *
 *     gsl_driver <deck dir> <t_stop> <cluster> <out file>
 *
 * Output file (binary, native doubles): nx, t, h, rhs_calls, accepted, rejected,
 * y[4 nx] at the end, dydt[4 nx] = sys.function(t, y) at the end (one more RHS
 * call through the struct, with the reference's side effects), then the breaking
 * log length L and its L doubles (hw_breaking_log's records).
 */
#include <stdio.h>
#include <stdlib.h>

#include "hawassi_b200.h"

/* the layout of GSL's gsl_odeiv_system */
typedef struct {
    int (*function)(double t, const double y[], double dydt[], void* params);
    int (*jacobian)(double t, const double y[], double* dfdy, double dfdt[], void* params);
    size_t dimension;
    void* params;
} gsl_odeiv_system;

static int fail(const char* what, const hw_ctx* ctx) {
    fprintf(stderr, "%s: %s\n", what, hw_last_error(ctx));
    return 1;
}

int main(int argc, char** argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s <deck> <t_stop> <cluster> <out>\n", argv[0]);
        return 2;
    }
    const char* deck = argv[1];
    const double t_stop = atof(argv[2]);
    hw_opts opts = {0};
    opts.cluster = atoi(argv[3]);
    hw_ctx* ctx = hw_create(deck, &opts);
    if (!ctx) return fail("hw_create", NULL);
    const int nx = hw_nx(ctx, 0), nt = hw_nt(ctx, 0);
    gsl_odeiv_system sys = {hw_gsl_rhs, NULL, (size_t)(4 * nx), ctx};

    double* tt = malloc(sizeof(double) * (size_t)nt);
    double* y = malloc(sizeof(double) * sys.dimension);
    double* dydt = malloc(sizeof(double) * sys.dimension);
    if (!tt || !y || !dydt) return 3;
    if (hw_deck_table(deck, &opts, "ttrace", tt, nt) < nt) return fail("hw_deck_table", NULL);
    if (hw_initial_state(ctx, 0, y)) return fail("hw_initial_state", ctx);

    double t = tt[0], h = 1e-4; /* the reference's first step (1d/functions.c:541) */
    for (int i = 1; i < nt && tt[i] <= t_stop; ++i) {
        while (t < tt[i]) {
            int status = hw_evolve_apply(ctx, 0, &t, tt[i], &h, y);
            if (status != 0) {
                fprintf(stderr, "error, return value=%d\n", status); /* 1d/functions.c:551 */
                return fail("hw_evolve_apply", ctx);
            }
        }
    }
    if (sys.function(t, y, dydt, sys.params) != 0) return fail("sys.function", ctx);

    long long rhs = 0, acc = 0, rej = 0, len = 0;
    int st = 0;
    if (hw_member_stats(ctx, 0, &rhs, &acc, &rej, &st)) return fail("hw_member_stats", ctx);
    if (hw_breaking_log(ctx, 0, NULL, 0, &len) < 0) return fail("hw_breaking_log", ctx);
    double* log = malloc(sizeof(double) * (size_t)(len > 0 ? len : 1));
    if (!log) return 3;
    if (len > 0 && hw_breaking_log(ctx, 0, log, len, &len) < 0) return fail("hw_breaking_log", ctx);

    FILE* f = fopen(argv[4], "wb");
    if (!f) return 4;
    double head[6] = {(double)nx, t, h, (double)rhs, (double)acc, (double)rej};
    double dl = (double)len;
    int ok = fwrite(head, sizeof(double), 6, f) == 6 && fwrite(y, sizeof(double), sys.dimension, f) == sys.dimension &&
             fwrite(dydt, sizeof(double), sys.dimension, f) == sys.dimension && fwrite(&dl, sizeof(double), 1, f) == 1 &&
             (len == 0 || fwrite(log, sizeof(double), (size_t)len, f) == (size_t)len);
    fclose(f);
    hw_destroy(ctx);
    free(tt);
    free(y);
    free(dydt);
    free(log);
    return ok ? 0 : 5;
}
