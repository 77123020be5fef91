"""B200 (sm_100a) implementation of the Lambda_b -> J/psi p K- unbinned amplitude likelihood.

Host-side mirror of the reference's model layer (model, configs), synthetic samples in the
reference's device layout (kinematics, basis, dataset) and the bindings of the CUDA library (lib).
"""
