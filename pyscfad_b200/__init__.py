"""pyscfad_b200: B200-native CCSD(T) perturbative-triples energy and VJP.

The compute path is the CUDA library built in-tree under pyscfad_b200/lib
(python -m pyscfad_b200._build); see include/pyscfad_b200.h for its C-ABI.
"""
__version__ = "0.1.0"
