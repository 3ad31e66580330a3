"""Oracle package: CPU restatement of the HERACLES++ MUSCL-Hancock step.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this package; the product library
``heraclespp_b200`` never does.
"""
from .pyoracle import Oracle, RefCell, RefStep, build_oracle, oracle_lib_path, ref_step_path, reference_root  # noqa: F401
