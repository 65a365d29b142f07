/*
 * spo_mlp.h - C ABI of the learned potential: a BF16 multilayer perceptron trained and evaluated on the
 * B200 tensor cores (tcgen05, FP32 accumulation in tensor memory).
 *
 * No counterpart in the reference, whose potential is evaluated exactly on the host (PotentialGrid,
 * src/potential/potential_grid.hpp:21-55). The network stands in for that evaluation on new grids: it
 * is trained on potential values the exact method produced (features -> V in hartree), then fills V
 * for other points; the exact values remain the reference and the fallback.
 *
 * Network: n_in features (zero-padded to a multiple of 64) -> depth hidden layers of `width` units with
 * SiLU -> 1 output. Weights are kept in FP32 (Adam state too) and used as BF16 copies; activations are
 * BF16 between layers; every product accumulates in FP32.
 *
 * Conventions as in spo_b200.h: int status (SPO_OK = 0), messages through spo_mlp_last_error, host
 * pointers, synchronous calls.
 */
#ifndef SPO_MLP_H
#define SPO_MLP_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spo_mlp spo_mlp;

/* Network of n_in inputs (1..64), `depth` hidden layers (1..8) of `width` units (64, 128 or 256), one
 * output. Weights initialised from `seed` (uniform, fan-in scaled), biases zero. */
int spo_mlp_create(int n_in, int width, int depth, unsigned long long seed, int device, spo_mlp** out);
int spo_mlp_destroy(spo_mlp* m);
const char* spo_mlp_last_error(const spo_mlp* m);

/* Number of parameters (FP32): layer by layer, W (out x in, row-major, in = the padded input width for
 * the first layer) then b. */
int spo_mlp_parameter_count(const spo_mlp* m, long long* n);
int spo_mlp_get_parameters(spo_mlp* m, float* out);
int spo_mlp_set_parameters(spo_mlp* m, const float* in);
/* The padded input width (n_in rounded up to 64). */
int spo_mlp_input_width(const spo_mlp* m, int* n);

/* y[i] = network(x[i]) for n points, x row-major (n x n_in), FP32 in and out. */
int spo_mlp_predict(spo_mlp* m, const float* x, long long n, float* y);

/* Loss (mean squared error over the n points) and its gradient with respect to every parameter, in the
 * order of spo_mlp_get_parameters, for the current parameters. n <= 65536. */
int spo_mlp_gradients(spo_mlp* m, const float* x, const float* y, long long n, double* loss, float* grad);

/* Adam training (beta1 0.9, beta2 0.999, eps 1e-8) on n points for `epochs` passes in batches of `batch`
 * (a multiple of 128, at most 65536), the batch order shuffled per epoch from `seed`; the learning rate
 * decays by cosine from lr to lr/20 over the run. Returns the mean training loss of the last epoch. */
int spo_mlp_train(spo_mlp* m, const float* x, const float* y, long long n, int epochs, int batch, float lr,
                  unsigned long long seed, double* last_epoch_loss);

#ifdef __cplusplus
}
#endif

#endif /* SPO_MLP_H */
