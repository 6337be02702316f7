"""install_alias(): unchanged reference-style imports load this package's classes."""
import subprocess
import sys
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_module_names_resolve():
    code = (
        "import gw_fopt_b200\n"
        "gw_fopt_b200.install_alias()\n"
        "from gw_fopt.bubble_gw import many_bubbles\n"
        "import gw_fopt.bubble_gw.many_bubbles as m2\n"
        "from gw_fopt.bubble_gw._py_bubble_gw.many_bubbles import GeneralizedBulkFlow\n"
        "import gw_fopt_b200.many_bubbles as mb\n"
        "assert many_bubbles is mb and m2 is mb and GeneralizedBulkFlow is mb.GeneralizedBulkFlow\n"
        "from gw_fopt.bubble_gw import _py_bubble_gw\n"
        "try:\n"
        "    _py_bubble_gw.two_bubbles.anything\n"
        "    raise SystemExit('two_bubbles should raise')\n"
        "except AttributeError as e:\n"
        "    assert 'not provided' in str(e)\n"
        "gw_fopt_b200.install_alias()  # idempotent\n"
        "print('ok')\n"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"
