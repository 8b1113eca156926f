"""Bindings for frameworks that own device memory and streams (XLA / JAX)."""
