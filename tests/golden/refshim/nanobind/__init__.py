"""Stand-in for the `nanobind` package, used only to build the reference
simulator's generated wrapper when producing golden fixtures.

The reference's generated CMakeLists asks `python -m nanobind --cmake_dir`
for a directory holding `nanobind-config.cmake`; this package answers with
its own `cmake/` folder, whose config maps `nanobind_add_module` onto a plain
pybind11 module (see include/nanobind/nanobind.h).
"""
import os

def cmake_dir():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "cmake")
