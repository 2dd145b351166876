"""The C++ solver API (include/paxpro/paxpro.hpp) compiles warning-free and
links against the library; usage examples mirror the reference's
(Examples/waveguide2D.cpp pattern)."""
from tests.cpp_build import build


def test_cpp_examples_compile_and_link():
    for name in ("waveguide2d", "sphere3d"):
        assert build(name)
