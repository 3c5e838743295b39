"""CPU: the C++ adapters compile against the C header (no GPU needed)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_adapters_compile(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "memphys.hpp"\nint main(){memphys::PARAMETERS p; (void)p; return 0;}\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only",
                    "-I", os.path.join(ROOT, "memphys_b200", "host"), str(src)], check=True)
