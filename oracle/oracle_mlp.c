/*
 * oracle_mlp.c -- CPU restatement of the learned vertical-mixing closure's
 * network, part of the oracle (test infrastructure only: the GPU training
 * and inference kernels are checked against it; nothing in the product
 * calls it).
 *
 * The network stands in for d3_end (src/fv_mixing.F90:73-347) per node
 * column: IN = 3*NS + 3 inputs (per interface the squared shear, the
 * buoyancy frequency squared and the interface depth; then the surface
 * forcing term, the bottom friction term and the total depth, all
 * normalised), three hidden layers of 256 with SiLU, OUT = NS outputs
 * (log of the viscosity snu and of the diffusivity Kv per interface,
 * normalised).  Layer l computes Z_l = A_{l-1} W_l^T + b_l with W_l stored
 * row-major (out x in); the flat parameter vector is W1 b1 W2 b2 W3 b3 W4 b4.
 * The loss is the mean squared error over the batch and the outputs.
 *
 * Everything here accumulates in double: it is the reference the FP32
 * device kernels are held to, and its own gradients are checked against
 * central finite differences in the CPU tests.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MLP_H 256

static void mlp_dims(int NS, int d[5]) {
    d[0] = 3 * NS + 3;
    d[1] = MLP_H;
    d[2] = MLP_H;
    d[3] = MLP_H;
    d[4] = NS;
}

int64_t oracle_mlp_nparams(int NS) {
    int d[5];
    mlp_dims(NS, d);
    int64_t n = 0;
    for (int l = 0; l < 4; ++l) n += (int64_t)d[l + 1] * d[l] + d[l + 1];
    return n;
}

static double silu(double z) { return z / (1.0 + exp(-z)); }
static double silu_grad(double z) {
    const double s = 1.0 / (1.0 + exp(-z));
    return s * (1.0 + z * (1.0 - s));
}

/* forward pass of B samples; Z[l] (pre-activations) and A[l] (activations,
 * A[0] = X) are kept for the backward pass when non-NULL */
static void forward(int NS, const float *p, const float *X, int B, double **Z, double **A, double *Y) {
    int d[5];
    mlp_dims(NS, d);
    const float *w = p;
    const double *in = NULL;
    double *a0 = A[0];
    for (int i = 0; i < B * d[0]; ++i) a0[i] = X[i];
    in = a0;
    for (int l = 0; l < 4; ++l) {
        const int ni = d[l], no = d[l + 1];
        const float *W = w, *b = w + (size_t)no * ni;
        double *z = (l < 3) ? Z[l + 1] : Y;
        for (int s = 0; s < B; ++s)
            for (int o = 0; o < no; ++o) {
                double acc = b[o];
                for (int k = 0; k < ni; ++k) acc += (double)W[(size_t)o * ni + k] * in[(size_t)s * ni + k];
                z[(size_t)s * no + o] = acc;
            }
        if (l < 3) {
            double *a = A[l + 1];
            for (int i = 0; i < B * no; ++i) a[i] = silu(z[i]);
            in = a;
        }
        w += (size_t)no * ni + no;
    }
}

static int alloc_acts(int NS, int B, double **Z, double **A) {
    int d[5];
    mlp_dims(NS, d);
    for (int l = 0; l < 4; ++l) {
        A[l] = malloc(sizeof(double) * (size_t)B * d[l]);
        Z[l] = malloc(sizeof(double) * (size_t)B * d[l]);
        if (!A[l] || !Z[l]) return 1;
    }
    return 0;
}

static void free_acts(double **Z, double **A) {
    for (int l = 0; l < 4; ++l) {
        free(A[l]);
        free(Z[l]);
    }
}

/* Y[B x OUT] = network(X[B x IN]) */
int oracle_mlp_forward(int NS, const float *params, const float *X, int B, float *Y) {
    int d[5];
    mlp_dims(NS, d);
    double *Z[4], *A[4];
    double *y = malloc(sizeof(double) * (size_t)B * d[4]);
    if (alloc_acts(NS, B, Z, A) || !y) return 1;
    forward(NS, params, X, B, Z, A, y);
    for (int i = 0; i < B * d[4]; ++i) Y[i] = (float)y[i];
    free(y);
    free_acts(Z, A);
    return 0;
}

/* loss = mean((Y - T)^2) over B x OUT, and its gradient with respect to
 * every parameter (same flat layout as params) */
int oracle_mlp_grad(int NS, const float *params, const float *X, const float *T, int B, double *loss, double *grads) {
    int d[5];
    mlp_dims(NS, d);
    double *Z[4], *A[4];
    const int out = d[4];
    double *y = malloc(sizeof(double) * (size_t)B * out);
    if (alloc_acts(NS, B, Z, A) || !y) return 1;
    forward(NS, params, X, B, Z, A, y);
    const double scale = 1.0 / ((double)B * out);
    double l2 = 0.0;
    /* delta of the output layer: dL/dZ4 = 2 (Y - T) / (B OUT) */
    double *delta = malloc(sizeof(double) * (size_t)B * MLP_H);
    double *dprev = malloc(sizeof(double) * (size_t)B * MLP_H);
    for (int i = 0; i < B * out; ++i) {
        const double r = y[i] - T[i];
        l2 += r * r;
        delta[i] = 2.0 * r * scale;
    }
    *loss = l2 * scale;
    /* offsets of each layer in the flat vector */
    size_t off[4];
    size_t o = 0;
    for (int l = 0; l < 4; ++l) {
        off[l] = o;
        o += (size_t)d[l + 1] * d[l] + d[l + 1];
    }
    for (int l = 3; l >= 0; --l) {
        const int ni = d[l], no = d[l + 1];
        const float *W = params + off[l];
        double *gW = grads + off[l], *gb = grads + off[l] + (size_t)no * ni;
        const double *ain = A[l];
        for (int oo = 0; oo < no; ++oo) {
            double sb = 0.0;
            for (int s = 0; s < B; ++s) sb += delta[(size_t)s * no + oo];
            gb[oo] = sb;
            for (int k = 0; k < ni; ++k) {
                double sw = 0.0;
                for (int s = 0; s < B; ++s) sw += delta[(size_t)s * no + oo] * ain[(size_t)s * ni + k];
                gW[(size_t)oo * ni + k] = sw;
            }
        }
        if (l > 0) {
            /* dL/dA_{l} = delta W_l, then through SiLU'(Z_l) */
            for (int s = 0; s < B; ++s)
                for (int k = 0; k < ni; ++k) {
                    double acc = 0.0;
                    for (int oo = 0; oo < no; ++oo) acc += delta[(size_t)s * no + oo] * (double)W[(size_t)oo * ni + k];
                    dprev[(size_t)s * ni + k] = acc * silu_grad(Z[l][(size_t)s * ni + k]);
                }
            double *t = delta;
            delta = dprev;
            dprev = t;
        }
    }
    free(delta);
    free(dprev);
    free(y);
    free_acts(Z, A);
    return 0;
}

/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) at step t >= 1 */
void oracle_mlp_adam(int64_t n, float *params, const double *grads, double *mom, double *var, int t, double lr) {
    const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
    const double c1 = 1.0 - pow(b1, t), c2 = 1.0 - pow(b2, t);
    for (int64_t i = 0; i < n; ++i) {
        mom[i] = b1 * mom[i] + (1.0 - b1) * grads[i];
        var[i] = b2 * var[i] + (1.0 - b2) * grads[i] * grads[i];
        const double mh = mom[i] / c1, vh = var[i] / c2;
        params[i] = (float)(params[i] - lr * mh / (sqrt(vh) + eps));
    }
}
