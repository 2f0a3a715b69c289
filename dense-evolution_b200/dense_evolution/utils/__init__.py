from .measurement import sample_counts, statevector_fidelity
