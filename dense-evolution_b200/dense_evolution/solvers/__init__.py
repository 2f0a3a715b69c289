from .autodiff import circuit_to_energy_fn
