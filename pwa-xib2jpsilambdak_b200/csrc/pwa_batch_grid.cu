// The smeared batched kernel for the weighted grid (Gaussian resolution).
#define PWA_NB 0
#define PWA_NB_NAME(x) x##_grid
#include "pwa_batch_nb.inc"
