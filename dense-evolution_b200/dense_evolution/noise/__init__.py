"""Noise for the dense statevector engine: the stochastic single-qubit Kraus
channels of the reference's ``dense_evolution.noise`` (``NoiseModel``) and the
noise configuration that ``energy_fn(noise=...)`` takes (``NoiseSpec``)."""
from .kraus_channels import MODELS, NoiseModel


class NoiseSpec:
    """A noise configuration for ``energy_fn(theta, h, noise=...)``: the model,
    its probability, the key that seeds the draws, and the target qubits
    (reference: ``dense_evolution/noise/differentiable.py``).  ``jax_key`` seeds
    the NumPy Generator the decisions are drawn from (an int, an array of ints
    or a Generator)."""

    def __init__(self, model: str, p, jax_key, qubits=None):
        self.model = model
        self.p = p
        self.jax_key = jax_key
        self.qubits = tuple(qubits) if qubits is not None else None

    def __repr__(self):
        return f"NoiseSpec(model={self.model!r}, p={self.p!r}, qubits={self.qubits!r})"


__all__ = ['NoiseModel', 'NoiseSpec', 'MODELS']
