// The smeared batched kernel for the 20-offset quantile scheme.
#define PWA_NB 20
#define PWA_NB_NAME(x) x##_20
#include "pwa_batch_nb.inc"
