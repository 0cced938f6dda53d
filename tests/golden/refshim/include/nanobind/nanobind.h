// nanobind API subset used by the reference's generated wrapper, expressed
// with pybind11. Each class is registered module-local: nanobind keeps one
// type domain per network (NB_DOMAIN) while pybind11's registry is global,
// so two networks in one process would otherwise clash.
#pragma once
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

namespace nanobind {
using pybind11::init;
using pybind11::overload_cast;

template <typename T, typename... Extra>
struct class_ : pybind11::class_<T, Extra...> {
  using Base = pybind11::class_<T, Extra...>;
  template <typename Mod>
  class_(Mod&& m, const char* name) : Base(std::forward<Mod>(m), name, pybind11::module_local()) {}
  template <typename... A> class_& def(A&&... a) { Base::def(std::forward<A>(a)...); return *this; }
  template <typename... A> class_& def_rw(A&&... a) { Base::def_readwrite(std::forward<A>(a)...); return *this; }
  template <typename... A> class_& def_ro(A&&... a) { Base::def_readonly(std::forward<A>(a)...); return *this; }
  template <typename... A> class_& def_prop_rw(A&&... a) { Base::def_property(std::forward<A>(a)...); return *this; }
  template <typename... A> class_& def_prop_ro(A&&... a) { Base::def_property_readonly(std::forward<A>(a)...); return *this; }
};
}  // namespace nanobind

#define NB_MODULE(name, m) PYBIND11_MODULE(name, m)
