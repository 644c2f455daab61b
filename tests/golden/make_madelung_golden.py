"""Golden Madelung potentials from the reference's own Ewald code
(gpaw/utilities/ewald.py, imported by file path from the reference checkout;
it needs only numpy and scipy).  Run in a container that has the reference:

    python tests/golden/make_madelung_golden.py [/path/to/reference]

Writes tests/golden/madelung.json (cells and values)."""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
    'GPAW_REFERENCE', os.path.join(HERE, '..', '..', '..', 'reference'))

spec = importlib.util.spec_from_file_location(
    'ref_ewald', os.path.join(REF, 'gpaw', 'utilities', 'ewald.py'))
ewald = importlib.util.module_from_spec(spec)
spec.loader.exec_module(ewald)

CELLS = [
    np.diag([10.0, 10.0, 10.0]),
    np.diag([6.0, 8.0, 11.0]),
    np.array([[5.0, 0.0, 0.0], [2.5, 4.33012701892, 0.0], [0.0, 0.0, 7.0]]),
    np.array([[4.0, 1.0, 0.5], [0.3, 5.0, 0.2], [0.7, -0.4, 6.0]]),
]
out = [{'cell': c.tolist(), 'madelung': float(ewald.madelung(c))}
       for c in CELLS]
with open(os.path.join(HERE, 'madelung.json'), 'w') as f:
    json.dump(out, f, indent=1)
print(json.dumps(out))
