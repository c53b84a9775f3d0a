// The plan entry points' handles (include/arrowmetal.h:1419-1420), shared by the plan evaluator
// (plan.cpp) and the sort server (server.cpp).
#pragma once

#include <string>
#include <vector>

#include "am_internal.h"

// A named table: columns of equal length, retained while the source lives.
struct am_plan_source_t {
  std::string name;
  std::vector<std::string> names;
  std::vector<am_array*> cols;
  int64_t rows = 0;
  ~am_plan_source_t() {
    for (am_array* c : cols) am::release(c);
  }
};

// A plan's result: named columns of `rows` rows, owned by the result.
struct am_plan_result_t {
  std::vector<std::string> names;
  std::vector<am_array*> cols;
  int64_t rows = 0;
  ~am_plan_result_t() {
    for (am_array* c : cols) am::release(c);
  }
};
