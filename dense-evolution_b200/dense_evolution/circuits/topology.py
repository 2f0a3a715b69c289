"""Entangling-layer topologies (the reference's ``circuits/topology.py:17-79``)."""

VALID_PATTERNS = ('linear', 'circular', 'full', 'star', 'brick')


def entangling_layer(n_qubits, pattern='linear', gate='cx', reverse=False, hub=0):
    """Two-qubit gate tuples over `n_qubits` wired as `pattern`:
    linear (q, q+1); circular (+ (n-1, 0) when n > 2); full (all i < j);
    star (hub, q); brick (even pairs, then odd pairs)."""
    if n_qubits < 2:
        raise ValueError(f"entangling_layer needs at least 2 qubits, got {n_qubits}")
    if pattern not in VALID_PATTERNS:
        raise ValueError(f"unknown pattern {pattern!r}, expected one of {VALID_PATTERNS}")
    if pattern in ('linear', 'circular'):
        edges = [(q, q + 1) for q in range(n_qubits - 1)]
        if pattern == 'circular' and n_qubits > 2:
            edges.append((n_qubits - 1, 0))
    elif pattern == 'full':
        edges = [(i, j) for i in range(n_qubits) for j in range(i + 1, n_qubits)]
    elif pattern == 'star':
        if not 0 <= hub < n_qubits:
            raise ValueError(f"hub={hub} out of range for n_qubits={n_qubits}")
        edges = [(hub, q) for q in range(n_qubits) if q != hub]
    else:
        edges = [(q, q + 1) for q in range(0, n_qubits - 1, 2)] + [(q, q + 1) for q in range(1, n_qubits - 1, 2)]
    if reverse:
        edges = [(b, a) for a, b in edges]
    return [(gate, a, b) for a, b in edges]
