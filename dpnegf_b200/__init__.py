"""B200-native NEGF transport core: drop-in for the dpnegf hot path.

The public modules mirror the reference package layout:

* ``dpnegf_b200.recursive_green_cal.recursive_gf`` -- block-tridiagonal RGF
* ``dpnegf_b200.surface_green.selfEnergy`` / ``surface_green`` -- Lopez-Sancho
* ``dpnegf_b200.device_property.DeviceProperty`` -- T(E), DOS, LDOS, G^<
* ``dpnegf_b200.lead_property.LeadProperty`` -- lead self-energies and Gamma
* ``dpnegf_b200.density.Ozaki`` -- pole-sum density

All numerical work runs in the CUDA library ``libnegf_b200.so`` built from
``dpnegf_b200/csrc`` (see ``dpnegf_b200/_lib.py``); there is no CPU fallback.
"""
__version__ = "0.1.0"
