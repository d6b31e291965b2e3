// tenes_gpu_main: one `tenes input.toml` run as a C call.
//
// The reference builds its driver into libtenes.so behind
//   extern "C" int tenes_itps_main(const char* input_filename, MPI_Comm comm,
//                                  int print_level)
// (src/iTPS/main.hpp:26-28, main.cpp:33-39), whose exceptions propagate to
// the caller.  Here the same run -- read the expert input file, simple /
// full update or time evolution, CTMRG, measurements, the output files in
// `outdir` -- is the library's front end (tenes_b200.itps), which drives the
// device through this library's C ABI.  This file embeds it: the CPython API
// is resolved at run time (the interpreter the process already runs, or
// libpython loaded on first use), so libtenes_gpu.so itself has no link-time
// dependency on Python.  Every failure comes back as a tg_status, with the
// message in tg_last_error(); nothing is thrown across the ABI.
#include <dlfcn.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "common.hpp"
#include "tenes_gpu.h"

#ifndef TG_PY_LIB
#define TG_PY_LIB "libpython3.so"
#endif
#ifndef TG_PY_SITE
#define TG_PY_SITE ""
#endif

namespace {

// The part of the CPython C API used below (stable ABI functions only).
struct PyApi {
  using Obj = void*;
  int (*IsInitialized)() = nullptr;
  void (*InitializeEx)(int) = nullptr;
  int (*GILState_Ensure)() = nullptr;  // PyGILState_STATE is an enum
  void (*GILState_Release)(int) = nullptr;
  void* (*Eval_SaveThread)() = nullptr;
  Obj (*Eval_GetBuiltins)() = nullptr;
  Obj (*Dict_New)() = nullptr;
  int (*Dict_SetItemString)(Obj, const char*, Obj) = nullptr;
  Obj (*Dict_GetItemString)(Obj, const char*) = nullptr;
  Obj (*Unicode_FromString)(const char*) = nullptr;
  const char* (*Unicode_AsUTF8)(Obj) = nullptr;
  Obj (*Long_FromLong)(long) = nullptr;
  long (*Long_AsLong)(Obj) = nullptr;
  Obj (*Run_String)(const char*, int, Obj, Obj) = nullptr;
  void (*Err_Print)() = nullptr;
  void (*DecRef)(Obj) = nullptr;
  bool ok = false;
};

constexpr int kPyFileInput = 257;  // Py_file_input

template <typename F>
bool bind(void* h, const char* name, F& f) {
  f = reinterpret_cast<F>(dlsym(h, name));
  return f != nullptr;
}

bool bind_all(void* h, PyApi& a) {
  return bind(h, "Py_IsInitialized", a.IsInitialized) && bind(h, "Py_InitializeEx", a.InitializeEx) &&
         bind(h, "PyGILState_Ensure", a.GILState_Ensure) && bind(h, "PyGILState_Release", a.GILState_Release) &&
         bind(h, "PyEval_SaveThread", a.Eval_SaveThread) && bind(h, "PyEval_GetBuiltins", a.Eval_GetBuiltins) &&
         bind(h, "PyDict_New", a.Dict_New) && bind(h, "PyDict_SetItemString", a.Dict_SetItemString) &&
         bind(h, "PyDict_GetItemString", a.Dict_GetItemString) &&
         bind(h, "PyUnicode_FromString", a.Unicode_FromString) && bind(h, "PyUnicode_AsUTF8", a.Unicode_AsUTF8) &&
         bind(h, "PyLong_FromLong", a.Long_FromLong) && bind(h, "PyLong_AsLong", a.Long_AsLong) &&
         bind(h, "PyRun_String", a.Run_String) && bind(h, "PyErr_Print", a.Err_Print) &&
         bind(h, "Py_DecRef", a.DecRef);
}

std::mutex g_main_mu;
PyApi g_py;
std::string g_py_error;

// The interpreter to run the front end in: the process's own when it has one
// (the library loaded from Python), else libpython (TENES_GPU_LIBPYTHON, or
// the one the library was built against) initialised here once and kept.
bool python_api() {
  if (g_py.ok) return true;
  PyApi a;
  if (bind_all(RTLD_DEFAULT, a) && a.IsInitialized()) {
    a.ok = true;
    g_py = a;
    return true;
  }
  const char* env = std::getenv("TENES_GPU_LIBPYTHON");
  const char* lib = (env && *env) ? env : TG_PY_LIB;
  void* h = dlopen(lib, RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    g_py_error = std::string("cannot load the Python runtime ") + lib + ": " + dlerror() +
                 " (set TENES_GPU_LIBPYTHON to the path of libpython)";
    return false;
  }
  if (!bind_all(h, a)) {
    g_py_error = std::string("the Python runtime ") + lib + " lacks a required C API function";
    return false;
  }
  if (!a.IsInitialized()) {
    a.InitializeEx(0);  // no signal handlers: the host process keeps its own
    a.Eval_SaveThread();  // release the GIL; every call takes it with GILState_Ensure
  }
  a.ok = true;
  g_py = a;
  return true;
}

// Directory that holds the tenes_b200 package: two levels above this library
// (tenes_b200/libtenes_gpu.so).
std::string package_root() {
  Dl_info info{};
  if (!dladdr(reinterpret_cast<const void*>(&package_root), &info) || !info.dli_fname) return "";
  std::string p(info.dli_fname);
  for (int up = 0; up < 2; ++up) {
    const size_t s = p.find_last_of('/');
    if (s == std::string::npos) return ".";
    p = p.substr(0, s);
  }
  return p.empty() ? "/" : p;
}

const char* kDriver =
    "import sys\n"
    "if py_site:\n"
    "    import site as _site\n"
    "    _site.addsitedir(py_site)\n"
    "if root not in sys.path:\n"
    "    sys.path.insert(0, root)\n"
    "from tenes_b200.itps import run_status\n"
    "rc, msg = run_status(input_path, print_level)\n";

}  // namespace

extern "C" int tenes_gpu_main(const char* input_toml, int print_level) {
  std::lock_guard<std::mutex> lock(g_main_mu);
  try {
    if (!input_toml || !*input_toml) tg::fail(TG_E_INPUT, "input file name is empty");
    if (!python_api()) tg::fail(TG_E_RUNTIME, g_py_error);
    const PyApi& py = g_py;
    const int gil = py.GILState_Ensure();
    int rc = TG_E_RUNTIME;
    std::string msg = "the front end stopped with a Python error (traceback on stderr)";
    PyApi::Obj g = py.Dict_New();
    if (g) {
      const std::string root = package_root();
      const char* site_env = std::getenv("TENES_GPU_PYTHON_SITE");
      const char* site = (site_env && *site_env) ? site_env : TG_PY_SITE;
      auto set_str = [&](const char* k, const char* v) {
        PyApi::Obj o = py.Unicode_FromString(v);
        py.Dict_SetItemString(g, k, o);
        py.DecRef(o);
      };
      py.Dict_SetItemString(g, "__builtins__", py.Eval_GetBuiltins());
      set_str("input_path", input_toml);
      set_str("root", root.c_str());
      set_str("py_site", site);
      PyApi::Obj pl = py.Long_FromLong(print_level);
      py.Dict_SetItemString(g, "print_level", pl);
      py.DecRef(pl);
      PyApi::Obj r = py.Run_String(kDriver, kPyFileInput, g, g);
      if (!r) {
        py.Err_Print();
      } else {
        py.DecRef(r);
        PyApi::Obj c = py.Dict_GetItemString(g, "rc");
        PyApi::Obj m = py.Dict_GetItemString(g, "msg");
        if (c) rc = static_cast<int>(py.Long_AsLong(c));
        const char* ms = m ? py.Unicode_AsUTF8(m) : nullptr;
        msg = ms ? ms : "";
      }
      py.DecRef(g);
    }
    py.GILState_Release(gil);
    if (rc != TG_OK) tg::set_last_error(msg);
    return rc;
  } catch (const tg::Error& e) {
    tg::set_last_error(e.what());
    return e.code;
  } catch (...) {
    tg::set_last_error("unknown error");
    return TG_E_RUNTIME;
  }
}
