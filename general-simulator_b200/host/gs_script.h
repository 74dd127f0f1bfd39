// gs_script.h -- the script language of General-Simulator.
//
// Mirrors the reference's front end (src/input.cu, src/variable.cu,
// src/pub.h:24-26): lines of `command args`, `;` as a line break, `#`
// comments, `{expr}` and `shell` backtick substitution, `:name=expr`,
// `loop N`/`while expr`/`if expr`..`else`..`end` blocks.  The commands that
// touch fields and the physics are forwarded to the driver (gs_driver.h).
#pragma once
#include <string>

#include "gs_data.h"

namespace gsfe {

class Driver;

// Expression values: the reference keeps both the text and a double; every
// operator result is re-printed with six significant digits.
struct ExprResult {
  std::string text;
  double val = 0;
  int rc = kNormal;
};

class Expressions {
 public:
  Store<std::string> local;              // script variables (:a=3)
  Store<std::string>* globals = nullptr;  // the driver's `set` variables ($name)
  ExprResult eval(std::string expr);
  // replace `cmd` by its output and {expr} by its value (Variable::ReplaceExpr)
  int substitute(std::string& line);
  // evaluate a whole expression in place, {} read as () (Variable::Evaluate)
  int evaluate(std::string& expr);
  int shell(const std::string& cmd, std::string& out);
};

class Interpreter {
 public:
  explicit Interpreter(Driver& d);
  // comments, ';', blank squeezing inside () and splitting of {a, b} lists
  // (INPUT::standardize, src/input.cu:133-213)
  static void standardize(std::string& script);
  int run(std::string script);  // INPUT::Phrasing

 private:
  bool next_line(std::string& line, std::string& script);
  int block_loop(std::string args, std::string& script);
  int block_while(std::string args, std::string& script);
  int block_if(std::string args, std::string& script);
  int readhere(std::string args, std::string& script);
  Driver& drv_;
  Expressions& ex_;
};

}  // namespace gsfe
