"""``python -m sovereign_moe_b200 solve MODEL.mps ...`` (see ``cli.py``)."""

import sys

from .cli import main

sys.exit(main())
