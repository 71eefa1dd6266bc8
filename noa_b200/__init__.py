"""noa_b200: B200-native (sm_100a) Fourier central-slice extraction and insertion.

Drop-in for noa's ``noa::xform`` central-slice functions (noa/xform/FourierProject.hpp); see
``noa_b200.fourier_project`` for the host API and ``include/noa_b200/fourier_project.h`` for the C ABI.
"""
