"""mtb: B200-native W-projection imaging path of mt-imager.

``mtb.imager.WProjectionImager`` is the host API; ``mtb._lib`` binds the C ABI
of libmtb.so (include/mtb.h); ``mtb.synth`` makes seeded synthetic
observations in mt-imager's record layout.
"""
__version__ = "0.1.0"
