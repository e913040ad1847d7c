"""B200-native split-explicit ARW RK3 dycore step (wrf_gpu ``_rk_scan_step`` drop-in).

Hand-written sm_100a CUDA behind the C ABI of ``include/wrfgpu.h``; this
package holds the host-side mirror of the reference interface
(:mod:`wrf_gpu_b200.dycore`), the in-tree build (:mod:`wrf_gpu_b200.build`)
and synthetic input builders (:mod:`wrf_gpu_b200.cases`).
"""

__version__ = "0.1.0"
