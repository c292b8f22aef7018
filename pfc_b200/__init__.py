"""B200-native spectral relaxation of phase field crystal (PFC) density fields.

Drop-in for the hot path of petenez/pfc's pfc-relax: the semi-implicit (ETD1)
spectral step, the free-energy / mean-density evaluation and the box-size
optimisation, as hand-written sm_100a CUDA behind the C ABI in
include/pfc_b200.h (libpfc_b200.so). This package is the Python view of that
ABI (``pfc_b200.lib``) plus input generation and file formats.
"""
