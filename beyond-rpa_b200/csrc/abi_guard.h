// No C++ exception may cross the C ABI: a C or Fortran caller cannot unwind one, so an escaping
// std::bad_alloc (a host vector sized by the caller's dimensions, a plan map, an error string)
// would terminate the caller's process.  Every exported entry point is therefore a
// function-try-block whose handler turns the exception in flight into a status code here.
#pragma once

#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/rpa_b200.h"

namespace rpa {

// Call only from inside a catch handler.  Host allocation failures map to RPA_ERR_OOM, container
// length errors to RPA_ERR_TOO_LARGE, anything else to RPA_ERR_INTERNAL; the exception's text
// goes to *detail when one is given.
inline int status_of_exception(std::string* detail) noexcept {
  int status = RPA_ERR_INTERNAL;
  const char* what = "unknown exception";
  try {
    throw;
  } catch (const std::bad_alloc& e) {
    status = RPA_ERR_OOM;
    what = e.what();
  } catch (const std::length_error& e) {
    status = RPA_ERR_TOO_LARGE;
    what = e.what();
  } catch (const std::exception& e) {
    what = e.what();
  } catch (...) {
  }
  if (detail) {
    try {
      *detail = std::string("host exception: ") + what;
    } catch (...) {
    }
  }
  return status;
}

// Where an array argument lives, from the memory type and device that cudaPointerGetAttributes
// reports for it.  `type` is a cudaMemoryType value (0 unregistered host memory, 1 registered or
// pinned host memory, 2 device memory, 3 managed memory); `ptr_device` is the device of device
// memory.  Device memory of a GPU other than the handle's is refused before any launch: the
// kernels read device arguments in place, and a kernel of one GPU given another GPU's address
// would fault or read the wrong memory.  Managed memory is reachable from every GPU.
enum class ArgMemory { Host, HandleDevice, OtherDevice };

inline ArgMemory classify_arg_memory(int type, int ptr_device, int handle_device) noexcept {
  if (type == 2) return ptr_device == handle_device ? ArgMemory::HandleDevice : ArgMemory::OtherDevice;
  if (type == 3) return ArgMemory::HandleDevice;
  return ArgMemory::Host;
}

}  // namespace rpa
