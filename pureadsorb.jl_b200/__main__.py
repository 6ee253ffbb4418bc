"""`python pureadsorb.jl_b200 widom ...`: the command line of cli.py. The directory is run as a
script, so the package is first imported from it under the name pureadsorb_b200."""
import importlib.util
import os
import sys


def _package():
    name = "pureadsorb_b200"
    if name in sys.modules:
        return sys.modules[name]
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location(name, os.path.join(here, "__init__.py"),
                                                  submodule_search_locations=[here])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    _package()
    from pureadsorb_b200 import cli  # noqa: E402

    sys.exit(cli.main())
