// Host-side interface of the learned closure's network (k_mlp.cu): the
// training state on the device and the functions model.cu builds the C-ABI
// entry points from.  No counterpart in the reference.
#pragma once
#include <cstdint>
#include <vector>

#include "closure.h"
#include "fesomc_gpu.h"

namespace fesomc {

constexpr int FESOMC_ENOMEM_LC = FESOMC_ENOMEM;
constexpr int FESOMC_ECUDA_LC = FESOMC_ECUDA;
constexpr int FESOMC_EINVAL_LC = FESOMC_EINVAL;
constexpr int FESOMC_ESTATE_LC = FESOMC_ESTATE;

struct LcNet {
    int NS = 0, IN = 0, OUT = 0;
    int dims[5] = {};
    long long off[4] = {};        // offsets of W_l in the flat parameter vector (b_l follows W_l)
    long long np = 0;             // parameters
    float *params = nullptr, *grads = nullptr, *mom = nullptr, *var = nullptr;
    int adam_t = 0;
    int rules = 0;                // fallback rules (kLcRule*) the model applies with this network
    // statistics, W = max(IN, OUT)-strided: mu_x, sd_x, mu_y, sd_y, lo_x, hi_x
    float *stats = nullptr;
    std::vector<float> h_stats;
    long long n_train = 0;        // harvested columns the statistics cover
    double *dloss = nullptr;
    // batch buffers (Bmax rows): inputs, targets, pre-activations, activations, deltas
    int Bmax = 0;
    float *Xb = nullptr, *Tb = nullptr, *Z[4] = {}, *A[4] = {}, *Dl[4] = {}, *part = nullptr;
    // training set harvested from the plain closure: transformed, not normalised
    float *hx = nullptr, *hy = nullptr;
    long long hcap = 0;
    unsigned long long *hcount = nullptr;
    // BF16 weights for the tensor-core kernel (chunk-major operand layout),
    // valid after lc_tc_prepare until the parameters change
    uint16_t *wtc = nullptr;
    unsigned int *tc_err = nullptr;
    bool tc_ready = false;
    cudaStream_t stream = nullptr;
    std::vector<void *> allocs;
};

LcNet *lc_create(int NS, long long hcap, unsigned long long seed, int Bmax, cudaStream_t s, int *rc);
void lc_free(LcNet *n);
// Y (B x OUT) = network(X (B x IN)), normalised values, device arrays, FP32
int lc_forward(LcNet *n, const float *X, long long B, float *Y);
// the same over B columns in one pass (the model's step), activations in two
// B x 256 buffers, launched on stream s
int lc_forward_full(const LcNet *n, const float *X, long long B, float *Y, float *bufA, float *bufB, cudaStream_t s);
// loss of one batch (B <= Bmax, normalised device arrays) and its gradient in n->grads
int lc_grad(LcNet *n, const float *X, const float *T, int B, double *loss);
// normalisation and envelope from the harvested set
int lc_fit_stats(LcNet *n);
// epochs of Adam over the harvested set in minibatches of B; mean loss per epoch
int lc_train(LcNet *n, int epochs, int B, float lr, unsigned long long seed, float *losses);
// BF16 tensor-core inference (k_mlp_tc.cu): whether the network's size fits
// the kernel, the BF16 weight copies, and Y = network(X) on stream s
bool lc_tc_supported(const LcNet *n);
int lc_tc_prepare(LcNet *n);
int lc_forward_tc(const LcNet *n, const float *X, long long B, float *Y, cudaStream_t s);

}  // namespace fesomc
