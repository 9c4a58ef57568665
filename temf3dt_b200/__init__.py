"""B200-native FETD time-stepping hot path for TEMF3DT (FP64, sm_100a).

The compute path lives in ``libtemf_b200.so`` (C ABI: ``include/temf_b200.h``);
``temf3dt_b200.fetd`` is the host-side mirror of the reference's forward
driver, ``temf3dt_b200.meshio`` its file formats and ``temf3dt_b200.synth``
the seeded synthetic model generator.
"""
__version__ = "0.1.0"
