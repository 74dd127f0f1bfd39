// gs_script.cpp -- expression evaluation and the line interpreter.
//
// Behaviour follows the reference's front end (HEAD side): src/input.cu
// (Phrasing :14-108, getline :111-132, standardize :133-213, readhere
// :216-242, block commands :256-347, print :350-355) and src/variable.cu
// (ReplaceExpr :66-104, Evaluate :106-114, ExprTree::Init :126-214), with
// the `p=p++` hang of standardize fixed.
#include "gs_script.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <random>

#include "gs_driver.h"

namespace gsfe {

namespace {

constexpr double kNanVal = -9.9999e23;  // _NAN_Var

struct OpDef {
  const char* s;
  int level;
};
// operator table and binding levels of src/pub.h:24-26 (lower binds later);
// at one position a later entry of equal or lower level wins
const OpDef kOps[] = {{"+", 15}, {"-", 15}, {"*", 18}, {"/", 18}, {"^", 21}, {"<", 9}, {">", 9}, {"<=", 8},
                      {">=", 8}, {"==", 8}, {"!=", 8}, {"=", 6}, {"+=", 6}, {"-=", 6}, {"*=", 6}, {"/=", 6}};

// a word counts as a number when removing exponent markers, signs and the
// decimal point leaves only digits (variable.cu:15-26)
bool looks_numeric(std::string s) {
  static const char* marks[] = {"E+", "E-", "e+", "e-", "E", "e", "+", "-", "."};
  for (const char* m : marks) {
    size_t p;
    const std::string ms(m);
    while ((p = s.find(ms)) != std::string::npos) s.erase(p, ms.size());
  }
  for (char c : s)
    if (c < '0' || c > '9') return false;
  return true;
}

std::string fmt(double v) { return to_string6(v); }

}  // namespace

int Expressions::shell(const std::string& cmd, std::string& out) {
  static std::mt19937 rng(12345u);
  const std::string tmp = ".gs.shell." + std::to_string(rng()) + ".tmp";
  const std::string full = cmd + " 2>&1 >" + tmp;
  if (std::system(full.c_str())) {
  }
  std::ifstream in(tmp);
  if (!in) {
    log() << "Error: fail to read shell results\n";
    return kNormal;
  }
  out.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  if (!out.empty()) out.erase(out.size() - 1);
  in.close();
  std::remove(tmp.c_str());
  return kNormal;
}

ExprResult Expressions::eval(std::string e) {
  ExprResult r;
  if (e.empty()) return r;
  {
    size_t p;
    while ((p = e.find(' ')) != std::string::npos) e.erase(p, 1);
  }
  while (e.size() >= 2 && e.front() == '(' && e.back() == ')') e = e.substr(1, e.size() - 2);
  const int len = (int)e.size();
  int depth = 0, pos = -1, op = -1, lev = 9999;
  for (int p = 0; p < len; ++p) {
    if (e[p] == '(') depth++;
    if (e[p] == ')') depth--;
    if (depth != 0) continue;
    if (p > 0 && (e[p] == '+' || e[p] == '-') && (e[p - 1] == 'e' || e[p - 1] == 'E')) continue;
    for (int i = 0; i < (int)(sizeof(kOps) / sizeof(kOps[0])); ++i) {
      const std::string o(kOps[i].s);
      if (e.compare(p, o.size(), o) == 0 && lev >= kOps[i].level) {
        pos = p;
        op = i;
        lev = kOps[i].level;
      }
    }
  }
  if (pos < 0) {
    std::string w = e;
    w = take_word(w);
    if (local.has(w)) {
      std::string v = local[w];
      r.text = take_word(v);
      r.val = to_real(r.text);
      return r;
    }
    if (!w.empty() && w[0] == '$') w.erase(0, 1);
    if (globals && globals->has(w)) {
      std::string v = (*globals)[w];
      r.text = take_word(v);
      r.val = to_real(r.text);
      return r;
    }
    if (looks_numeric(w)) {
      r.text = w;
      r.val = to_real(w);
      return r;
    }
    log() << "Error: \"" << w << "\" unknown \n";
    r.text = "nan";
    r.val = kNanVal;
    r.rc = kErr;
    return r;
  }
  const std::string o(kOps[op].s);
  const std::string L = e.substr(0, pos), R = e.substr(pos + o.size());
  const ExprResult right = eval(R);
  ExprResult left;
  if (o != "=") left = eval(L);
  if (left.text == "nan" || right.text == "nan") {
    r.text = "nan";
    r.val = kNanVal;
    return r;
  }
  const double a = left.val, b = right.val;
  if (o == "+") {
    r.val = a + b;
  } else if (o == "-") {
    r.val = a - b;
  } else if (o == "*") {
    r.val = a * b;
  } else if (o == "/") {
    if (b == 0) {
      r.text = "nan";
      r.val = kNanVal;
      return r;
    }
    r.val = a / b;
  } else if (o == "^") {
    // integer power by repeated float multiplication (Real ^ int)
    float acc = 1.0f, base = (float)a;
    for (int i = 1; i <= (int)b; ++i) acc = acc * base;
    r.val = acc;
  } else if (o == "<=") {
    r.val = a <= b;
  } else if (o == ">=") {
    r.val = a >= b;
  } else if (o == "==") {
    r.val = a == b;
  } else if (o == "!=") {
    r.val = a != b;
  } else if (o == "<") {
    r.val = a < b;
  } else if (o == ">") {
    r.val = a > b;
  } else if (o == "=") {
    if (L.empty() || L[0] != '$')
      local[L] = right.text;
    else if (globals)
      (*globals)[L.substr(1)] = right.text;
    r.text = right.text;
    r.val = right.val;
    return r;
  } else {
    // a op= b  ->  a = a op b
    return eval(L + "=" + L + o.substr(0, 1) + R);
  }
  r.text = fmt(r.val);
  return r;
}

int Expressions::substitute(std::string& s) {
  size_t l;
  while ((l = s.find('`')) != std::string::npos) {
    const size_t r = s.find('`', l + 1);
    if (r == std::string::npos) {
      log() << "Error: uncomplete expression\n";
      return kErr;
    }
    std::string out;
    const int rc = shell(s.substr(l + 1, r - l - 1), out);
    if (rc < 0) return rc;
    s.replace(l, r - l + 1, out);
  }
  while ((l = s.find('{')) != std::string::npos) {
    size_t r = std::string::npos;
    for (;;) {
      r = s.find('}', r == std::string::npos ? 0 : r + 1);
      if (r == std::string::npos) {
        log() << "Error: uncomplete expression\n";
        return kErr;
      }
      const size_t pl = s.find('{', l + 1);
      if (pl == std::string::npos || pl > r) break;
    }
    const ExprResult v = eval(s.substr(l + 1, r - l - 1));
    if (v.rc < 0) return v.rc;
    s.replace(l, r - l + 1, v.text);
  }
  return kNormal;
}

int Expressions::evaluate(std::string& e) {
  for (char& c : e) {
    if (c == '{') c = '(';
    if (c == '}') c = ')';
  }
  e = eval(e).text;
  return kNormal;
}

// ---------------------------------------------------------------------------

Interpreter::Interpreter(Driver& d) : drv_(d), ex_(d.expr) {}

void Interpreter::standardize(std::string& s) {
  s += "\n";
  for (char& c : s)
    if (c == ';') c = '\n';
  size_t p1;
  while ((p1 = s.find('#')) != std::string::npos) {
    const size_t p2 = s.find('\n', p1);
    s.erase(p1, p2 == std::string::npos ? std::string::npos : p2 - p1);
  }
  // an expression in parentheses loses its blanks and the parentheses
  int depth = 0;
  size_t pre = 0;
  for (size_t pos = 0; pos < s.size(); ++pos) {
    if (s[pos] == '(') {
      if (++depth == 1) pre = pos;
    } else if (s[pos] == ')') {
      if (--depth == 0) {
        std::string t = s.substr(pre + 1, pos - pre - 1);
        std::string u;
        for (char c : t)
          if (c != ' ' && c != '\n') u += c;
        s.replace(pre, pos - pre + 1, u);
        pos = pre + u.size() - 1;
        if (u.empty()) pos = pre - (pre > 0 ? 1 : 0);
      }
    }
  }
  // {a, b c} -> {a} {b} {c}: each blank, newline or comma closes one
  // expression and opens the next
  depth = 0;
  for (size_t pos = 0; pos < s.size(); ++pos) {
    if (s[pos] == '{') {
      if (++depth == 1) pre = pos;
    } else if (s[pos] == '}') {
      if (--depth == 0) {
        std::string t = s.substr(pre, pos - pre + 1);
        size_t q = 0;
        while (q < t.size()) {
          if (t[q] == ' ' || t[q] == '\n' || t[q] == ',') {
            t.replace(q, 1, "} {");
            q += 3;
            continue;
          }
          ++q;
        }
        s.replace(pre, pos - pre + 1, t);
        pos = pre + t.size() - 1;
      }
    }
  }
}

bool Interpreter::next_line(std::string& line, std::string& script) {
  if (script.empty()) return false;
  size_t n = script.find('\n');
  if (n == std::string::npos) n = script.size();
  line = script.substr(0, n);
  script.erase(0, n + 1);
  std::string first;
  (void)(line >>= first);
  if (first != "print") {
    ex_.substitute(line);
    for (char& c : line)
      if (c == ',') c = ' ';
  }
  if (!line.empty() && log().on) log() << ">>>" << line << "\n";
  return true;
}

namespace {
const char* kBlockWords[] = {"if", "loop", "while"};

// text up to the `end` that closes the block; every occurrence of if, loop,
// while opens a level and every `end` closes one (src/input.cu:256-272)
int split_block(std::string& script, std::string& body) {
  int open = 1;
  for (size_t p = 0; p < script.size(); ++p) {
    for (const char* w : kBlockWords)
      if (script.compare(p, std::string(w).size(), w) == 0) open++;
    if (script.compare(p, 3, "end") == 0) open--;
    if (open == 0) {
      body = script.substr(0, p);
      script.erase(0, p + 3);
      return kNormal;
    }
  }
  return kIncomplete;
}

int split_if(std::string& script, std::string& yes, std::string& no) {
  int open = 1;
  long p_else = -1, p_end = -1;
  for (size_t p = 0; p < script.size(); ++p) {
    for (const char* w : kBlockWords)
      if (script.compare(p, std::string(w).size(), w) == 0) open++;
    if (script.compare(p, 3, "end") == 0) open--;
    if (p_else < 0 && open == 1 && script.compare(p, 4, "else") == 0) p_else = (long)p;
    if (open == 0) {
      p_end = (long)p;
      break;
    }
  }
  if (open > 0) return kIncomplete;
  if (p_else < 0) {
    yes = script.substr(0, p_end);
    no.clear();
  } else {
    yes = script.substr(0, p_else);
    no = script.substr(p_else + 4, p_end - p_else - 4);
  }
  script.erase(0, p_end + 3);
  return kNormal;
}
}  // namespace

int Interpreter::block_loop(std::string args, std::string& script) {
  std::string count = take_word(args);
  script = args + "\n" + script;
  std::string body;
  split_block(script, body);
  ex_.evaluate(count);
  const double n = to_real(count);
  for (int i = 0; i < n; ++i) {
    const int rc = run(body);
    if (rc != kNormal) return rc;
  }
  return kNormal;
}

int Interpreter::block_while(std::string args, std::string& script) {
  std::string rest = args;
  std::string cond = take_word(rest);
  script = rest + "\n" + script;
  std::string body;
  split_block(script, body);
  ex_.evaluate(cond);
  while (to_real(cond) > 0) {
    const int rc = run(body);
    if (rc != kNormal) return rc;
    (void)(args >>= cond);
    ex_.evaluate(cond);
  }
  return kNormal;
}

int Interpreter::block_if(std::string args, std::string& script) {
  std::string cond = take_word(args);
  script = args + "\n" + script;
  std::string yes, no;
  split_if(script, yes, no);
  ex_.evaluate(cond);
  return run(to_real(cond) > 0 ? yes : no);
}

int Interpreter::readhere(std::string args, std::string& script) {
  const std::string name = take_word(args);
  std::string arrays, ln;
  long ndim = 1, nele = 1, index = 0;
  while (next_line(ln, script)) {
    while (!ln.empty()) {
      if (index == 0) {
        ln >> ndim;
        arrays += std::to_string(ndim) + " ";
      } else if (index <= ndim) {
        long t = 0;
        ln >> t;
        arrays += std::to_string(t) + " ";
        nele *= t;
      } else {
        arrays += take_word(ln) + " ";
      }
      index++;
    }
    if (index > ndim + nele) break;
  }
  return drv_.readhere(name, arrays);
}

int Interpreter::run(std::string script) {
  std::string ss;
  while (next_line(ss, script)) {
    const std::string line = ss;
    const size_t b = ss.find_first_not_of(' ');
    if (b == std::string::npos) continue;
    ss.erase(0, b);
    std::string cmd = take_word(ss);
    if (!cmd.empty() && cmd[0] == ':') {
      ss = cmd.substr(1) + " " + ss;
      cmd = "expr";
    }
    int err = kNormal;
    if (cmd == "expr") {
      err = ex_.evaluate(ss);
    } else if (cmd == "shell") {
      std::string out;
      err = ex_.shell(ss, out);
      log() << out << "\n";
    } else if (cmd == "log") {
      log().on = true;
    } else if (cmd == "break") {
      break;
    } else if (cmd == "quit") {
      err = kQuit;
      break;
    } else if (cmd == "link") {
      err = drv_.link(ss);
    } else if (cmd == "info") {
      err = drv_.set_info(ss);
    } else if (cmd == "dump") {
      err = drv_.set_dump(ss);
    } else if (cmd == "set") {
      err = drv_.set(ss);
    } else if (cmd == "read") {
      err = drv_.read(ss);
    } else if (cmd == "readhere") {
      err = readhere(ss, script);
    } else if (cmd == "write") {
      err = drv_.write(ss);
    } else if (cmd == "writehere") {
      err = drv_.writehere(ss);
    } else if (cmd == "device") {
      err = drv_.device(ss);
    } else if (cmd == "print") {
      err = ex_.substitute(ss);
      log() << ss << "\n";
    } else if (cmd == "sys") {
      err = drv_.set_sys(ss);
    } else if (cmd == "run") {
      err = drv_.run(ss);
    } else if (cmd == "loop") {
      err = block_loop(ss, script);
    } else if (cmd == "while") {
      err = block_while(ss, script);
    } else if (cmd == "if") {
      err = block_if(ss, script);
    } else if (cmd == "runfunc") {
      err = drv_.runfunc(ss);
    } else {
      err = drv_.runfunc(cmd + " " + ss);
    }
    if (err == kUnknown) {
      log() << "Error: " << line << " unknown\n";
      return kErr;
    }
    if (err == kErr) {
      log() << "Error: error in command \"" << line << "\"\n";
      return kErr;
    }
    if (err == kQuit) return kQuit;
  }
  return kNormal;
}

}  // namespace gsfe
