// cnn.cuh -- internal interface of the learned Poisson warm start (cnn.cu).
#pragma once
#include "lepic_internal.cuh"

#define CNN_LAYERS 12       // e0a e0b e1a e1b e2a e2b e3a e3b d2 d1 d0 out
#define CNN_MAX_BATCH 8     // training crops per step

struct CnnNet;
int cnn_net_create(CnnNet **out, int dev, cudaStream_t stream, unsigned long long seed);
void cnn_net_destroy(CnnNet *net);
int learned_solve(lepic_ctx *c, double eps);
int learned_stats(lepic_ctx *c, lepic_cnn_stats *out);
int learned_configure(lepic_ctx *c, const lepic_cnn_config *cfg);
void learn_free(lepic_ctx *c);
