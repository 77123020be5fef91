// The smeared batched kernel for the 150-offset quantile scheme.
#define PWA_NB 150
#define PWA_NB_NAME(x) x##_150
#include "pwa_batch_nb.inc"
