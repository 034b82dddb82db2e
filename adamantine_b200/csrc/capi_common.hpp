// Shared pieces of the extern "C" entry points: the exception-to-status
// guard and the per-thread error message.
#pragma once

#include "thermal.hpp"

#include <new>
#include <string>

namespace adm
{
void set_last_error(std::string const &msg);

// Runs f; returns ADM_OK, or the status of the exception it threw after
// recording the message for adm_last_error(). Nothing crosses the ABI.
template <class F>
int guard(F &&f)
{
  try
  {
    f();
    return ADM_OK;
  }
  catch (Error const &e)
  {
    set_last_error(e.what());
    return e.code;
  }
  catch (std::bad_alloc const &)
  {
    set_last_error("host allocation failed");
    return ADM_ERR_ALLOC;
  }
  catch (std::exception const &e)
  {
    set_last_error(e.what());
    return ADM_ERR_INVALID;
  }
  catch (...)
  {
    set_last_error("unknown error");
    return ADM_ERR_INVALID;
  }
}
} // namespace adm

#define ADM_REQUIRE(cond, msg)                                                 \
  do                                                                           \
  {                                                                            \
    if (!(cond))                                                               \
      throw adm::Error(ADM_ERR_INVALID, msg);                                  \
  } while (0)
