"""python -m pypaswas_b200 [options] FILE_1 FILE_2 -- the pyPaSWAS command line
(pypaswas.py) on the B200 engine; see pypaswas_b200.cli."""
import sys

from .cli import main

sys.exit(main())
