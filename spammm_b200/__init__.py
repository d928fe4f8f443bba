"""sm_100a implementation of SPAMMM's probe-particle AFM hot path.

``spammm_b200.AFM`` / ``spammm_b200.AFM_utils`` mirror ``spammm.SPM.AFM`` /
``spammm.SPM.AFM_utils`` for this path; ``spammm_b200.gpu`` holds the
device-resident tensor calls; the kernels live in ``libspmb200.so`` (C ABI:
include/spm_b200.h).
"""
__version__ = "0.1.0"
