"""``python -m pf_kks_gpu CONFIG --out DIR ...``: the ``pf-kks-run`` command."""

from .cli import entry

entry()
