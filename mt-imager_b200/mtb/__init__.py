"""mtb: B200-native W-projection imaging path of mt-imager.

``mtb.imager.WProjectionImager`` is the host API; ``mtb.lsrk`` converts the
channel frequencies TOPO -> LSRK per record from the TIME column;
``mtb.ingest`` reads record files in the baseline-major order; ``mtb.engine``
serves many imaging requests on one GPU; ``mtb._lib`` binds the C ABI of
libmtb.so (include/mtb.h); ``mtb.synth`` makes seeded synthetic observations
in mt-imager's record layout.
"""
__version__ = "0.1.0"
