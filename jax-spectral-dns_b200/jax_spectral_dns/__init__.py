"""B200-native velocity-vorticity channel-flow step with the reference's
Domain / Field / equation-class surface (dakling/jax-spectral-dns)."""
__version__ = "0.1.0"
