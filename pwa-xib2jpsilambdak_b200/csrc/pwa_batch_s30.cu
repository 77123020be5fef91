// The smeared batched kernel for the 30-offset quantile scheme.
#define PWA_NB 30
#define PWA_NB_NAME(x) x##_30
#include "pwa_batch_nb.inc"
