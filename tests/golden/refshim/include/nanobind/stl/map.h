#pragma once
// STL casters come from pybind11/stl.h (included by nanobind.h).
