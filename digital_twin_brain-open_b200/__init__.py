"""B200 engine for the Digital Twin Brain per-timestep hot path.

Submodules:
* ``engine``   -- ctypes binding of the C-ABI (include/dtb_b200.h), one network per Engine;
* ``network``  -- synthetic network specs and the small host-side generators;
* ``build``    -- nvcc recipe for the in-tree ``libdtb_b200.so``.

The directory name is not a Python identifier; load it as ``dtb_b200`` with
``__graft_entry__.load_package()`` (or any importlib loader that sets
``submodule_search_locations`` to this directory).
"""
__version__ = "1.0.0"
