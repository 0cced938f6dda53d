# Minimal nanobind package config: builds the wrapper as a pybind11 module.
# ANB_PYBIND11_INCLUDE must point at pybind11's include directory.
set(nanobind_FOUND TRUE)
get_filename_component(_anb_shim_inc "${CMAKE_CURRENT_LIST_DIR}/../../include" ABSOLUTE)
function(nanobind_add_module name)
  cmake_parse_arguments(ARG "" "NB_DOMAIN" "" ${ARGN})
  add_library(${name} MODULE ${ARG_UNPARSED_ARGUMENTS})
  set_target_properties(${name} PROPERTIES PREFIX "" POSITION_INDEPENDENT_CODE ON)
  target_include_directories(${name} PRIVATE ${_anb_shim_inc} $ENV{ANB_PYBIND11_INCLUDE} ${Python_INCLUDE_DIRS})
  target_compile_features(${name} PRIVATE cxx_std_17)
endfunction()
