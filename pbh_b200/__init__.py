"""pbh_b200: B200-native particle-mesh engine for the pm3d path of uniquehuman/pbh.

``pbh_b200.pm3d`` is the drop-in module (PM3D, analyse, zeldovich_axes, H_I, T_I, RHO_A3);
``pbh_b200.engine`` is the handle over the native library; ``pbh_b200.batch`` and
``pbh_b200.serve`` run ensembles and the request loop on one GPU.
"""
__version__ = "0.1.0"
