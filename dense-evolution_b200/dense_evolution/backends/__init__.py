from .statevector import DenseSVSimulator
