"""CPU: the C++ adapters compile against the C header (no GPU needed)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_adapters_compile(tmp_path):
    src = tmp_path / "t.cpp"
    # every adapter is instantiated (syntax and type check only: nothing runs)
    src.write_text('#include "memphys.hpp"\n'
                   'using namespace memphys;\n'
                   'void use(POINTS &pt, CLOUD &c, PARAMETERS &p, std::vector<bool> &f,\n'
                   '         std::vector<double> &a, std::vector<int> &l) {\n'
                   '  SEMI_IMPLICIT_SPLIT_SOLVER s(pt, c, p, f, f, f, 3, 1e-6, 1);\n'
                   '  s.single_timestep_2d(pt, c, p, a, a, a, a, a, a, 0, l, a, a);\n'
                   '  IMPLICIT_SCALAR_TRANSPORT_SOLVER t(pt, c, p, f, 1, 1.0, 1.0, -0.01, true);\n'
                   '  t.single_timestep_2d(pt, c, p, a, a, a, a, 0);\n'
                   '  FRACTIONAL_STEP_FOURIER q(pt, c, p, f, f, f, f, 1.0, 2, 2);\n'
                   '  q.single_timestep(pt, c, p, a, a, a, a, a, a, a, a, 0);\n'
                   '  INTERP_MATRIX m = calc_interp_matrix(a, pt, p); (void)m;\n'
                   '}\n'
                   'int main(){PARAMETERS p; (void)p; return 0;}\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only",
                    "-I", os.path.join(ROOT, "memphys_b200", "host"), str(src)], check=True)


def test_cpp_adapters_link_against_the_library(tmp_path):
    """A program using every adapter links against libmemphys_cuda.so (nothing runs:
    the CUDA driver library is resolved only at run time)."""
    from memphys_b200 import build
    lib = build.build()
    src = tmp_path / "link.cpp"
    src.write_text('#include "memphys.hpp"\n'
                   'using namespace memphys;\n'
                   'int main(int argc, char **) {\n'
                   '  if (argc > 99) {\n'
                   '    PARAMETERS p; POINTS pt; CLOUD c(pt, p);\n'
                   '    std::vector<bool> f; std::vector<double> a; std::vector<int> l;\n'
                   '    SEMI_IMPLICIT_SPLIT_SOLVER s(pt, c, p, f, f, f, 3, 1e-6, 1);\n'
                   '    s.single_timestep_2d(pt, c, p, a, a, a, a, a, a, 0, l, a, a);\n'
                   '    IMPLICIT_SCALAR_TRANSPORT_SOLVER t(pt, c, p, f, 1, 1.0, 1.0, -0.01, true);\n'
                   '    t.single_timestep_2d(pt, c, p, a, a, a, a, 0);\n'
                   '    FRACTIONAL_STEP_FOURIER q(pt, c, p, f, f, f, f, 1.0, 2, 2);\n'
                   '    q.single_timestep(pt, c, p, a, a, a, a, a, a, a, a, 0);\n'
                   '    FRACTIONAL_STEP_1 fs(pt, c, p, f, f, f, 2);\n'
                   '    INTERP_MATRIX m = calc_interp_matrix(a, pt, p); (void)m;\n'
                   '  }\n'
                   '  return 0;\n'
                   '}\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "memphys_b200", "host"), str(src),
                    "-L", os.path.dirname(lib), "-lmemphys_cuda", "-Wl,--allow-shlib-undefined",
                    "-o", str(tmp_path / "link")], check=True)
