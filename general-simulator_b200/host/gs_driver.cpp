// gs_driver.cpp -- GS: system registry, variables, field I/O and the run loop
// (src/gs.cu:20-227).  Differences from the reference, on purpose:
// BinaryMode / InfoSteps / DumpSteps start at off / 0 / 0 (the reference
// leaves them uninitialised); a failing Initialize stops `run`; fields are
// synchronised from the device before they are dumped or written (the
// reference writes the stale host copy of fields that were `read`).
#include "gs_driver.h"

#include <cstdlib>

#include "../../include/gs_capi.h"

namespace gsfe {

Log& log() {
  static Log l;
  return l;
}

Driver::Driver() { expr.globals = &vars; }

Dynamics* Driver::current() {
  auto it = systems_.find(name_);
  return it == systems_.end() ? nullptr : it->second.get();
}

int Driver::set_sys(std::string args) {
  const std::string sys = take_word(args);
  if (systems_.count(sys)) {
    name_ = sys;
    return kNormal;
  }
  std::unique_ptr<Dynamics> d = make_dynamics(sys);
  if (!d) {
    log() << "Error: unknown system \"" << sys << "\"\n";
    return kErr;
  }
  systems_[sys] = std::move(d);
  inited_[sys] = false;
  name_ = sys;
  return kNormal;
}

int Driver::set(std::string args) {
  const std::string var = take_word(args);
  if (var == "binary") {
    binary_ = take_word(args) == "on";
  } else if (var == "log") {
    log().on = take_word(args) != "off";
  } else {
    vars[var] = args;
  }
  return kNormal;
}

int Driver::link(std::string args) {
  const std::string target = take_word(args), alias = take_word(args);
  vars.link(target, alias);
  return kNormal;
}

int Driver::read(std::string args) {
  const std::string var = take_word(args), file = take_word(args);
  Field f;
  const bool ok = binary_ ? f.read_binary(file) : f.read_text(file);
  if (!ok) {
    std::cerr << "Error: \"" << file << "\" not found!\n";
    return kErr;
  }
  datas[var] = std::move(f);
  return kNormal;
}

int Driver::readhere(const std::string& name, std::string arrays) {
  long n = 0;
  arrays >> n;
  std::vector<int> dims(n > 0 ? n : 0);
  for (auto& d : dims) arrays >> d;
  Field f;
  f.init(dims);
  for (auto& x : f.v) arrays >> x;
  datas[name] = std::move(f);
  return kNormal;
}

void Driver::dump_field(const std::string& name, const std::string& file) {
  Field& f = datas[name];
  if (binary_)
    f.write_binary(file);
  else
    f.write_text(file);
}

int Driver::write(std::string args) {
  while (!args.empty()) {
    const std::string name = take_word(args);
    std::string file = take_word(args);
    if (name.empty()) break;
    if (Dynamics* d = current()) d->SyncToHost(name);
    if (datas.has(name)) {
      if (file.empty()) file = name + ".data";
      dump_field(name, file);
    } else {
      log() << "Error: unknown data \"" << name << "\"\n";
    }
  }
  return kNormal;
}

int Driver::writehere(std::string args) {
  while (!args.empty()) {
    const std::string name = take_word(args);
    if (name.empty()) break;
    if (Dynamics* d = current()) d->SyncToHost(name);
    if (datas.has(name)) {
      datas[name].print(std::cout);
      if (log().file) datas[name].print(log().file);
    } else if (vars.has(name)) {
      log() << vars[name];
    } else {
      log() << "Error: unknown data \"" << name << "\"\n";
    }
  }
  return kNormal;
}

int Driver::set_info(std::string args) {
  args >> info_steps_;
  info_mode_ = args;
  return kNormal;
}

int Driver::set_dump(std::string args) {
  dump_folder_ = take_word(args);
  args >> dump_steps_;
  const std::string cmd = "if [ -s " + dump_folder_ + " ]; then echo 'dump to folder" + dump_folder_ +
                          "'; else mkdir " + dump_folder_ + "; fi";
  if (std::system(cmd.c_str())) {
  }
  dump_mode_ = args;
  return kNormal;
}

void Driver::info_out() {
  Dynamics* d = current();
  std::string mode = info_mode_;
  log() << "Step  " << step_ << " \t";
  while (!mode.empty()) {
    const std::string key = take_word(mode);
    log() << d->Get(key) << " \t";
  }
  log() << "\n";
}

// Join the oldest asynchronous dumps until at most `keep` are in flight; the
// joined fields go into the store, as a synchronous dump leaves them.
int Driver::finish_dumps(size_t keep) {
  int rc = kNormal;
  while (pending_.size() > keep) {
    PendingDump p = std::move(pending_.front());
    pending_.pop_front();
    auto r = p.done.get();
    if (!r.first.empty()) {
      log() << "Error: dump of " << p.name << ": " << r.first << "\n";
      rc = kErr;
    } else {
      datas[p.name] = std::move(r.second);
    }
  }
  return rc;
}

void Driver::dump_out() {
  Dynamics* d = current();
  std::string mode = dump_mode_;
  std::string a;
  const bool async = !(vars.has("asyncdump") && (a = vars["asyncdump"], a == "0" || a == "off"));
  while (!mode.empty()) {
    const std::string name = take_word(mode);
    if (name.empty()) continue;
    const std::string file = dump_folder_ + "/" + name + "." + std::to_string(step_) + ".data";
    Dynamics::DumpJob job = async ? d->DumpAsync(name) : Dynamics::DumpJob();
    if (job) {
      // host memory stays bounded: at most two dumps wait for their writer
      finish_dumps(1);
      const bool binary = binary_;
      pending_.push_back({name, std::async(std::launch::async, [job, file, binary]() {
                            Field f;
                            std::string err = job(f);
                            if (err.empty() && !(binary ? f.write_binary(file) : f.write_text(file)))
                              err = "cannot write " + file;
                            return std::make_pair(err, std::move(f));
                          })});
      continue;
    }
    d->SyncToHost(name);
    if (datas.has(name)) {
      dump_field(name, file);
    } else {
      log() << "Error: data " << name << " does not exist!\n";
    }
  }
}

int Driver::run(std::string args) {
  Dynamics* d = current();
  if (!d) {
    log() << "Error: system not set\n";
    return kErr;
  }
  int total = 1;
  args >> total;
  if (total <= 0) return kErr;
  d->Datas = &datas;
  d->Vars = &vars;
  if (!inited_[name_]) {
    if (d->Initialize() != kNormal) return kErr;
    inited_[name_] = true;
    step_ = 0;
    (void)(vars["ahead_steps"] >>= step_);
  }
  int info_every = info_steps_ == 0 ? total + 1 : total / info_steps_;
  if (info_every == 0) info_every = 1;
  int dump_every = dump_steps_ == 0 ? total + 1 : total / dump_steps_;
  if (dump_every == 0) dump_every = 1;
  {
    std::string mode = info_mode_;
    log() << "Info \t\t";
    while (!mode.empty()) log() << take_word(mode) << "\t";
    log() << "\n";
  }
  for (int i = 1; i <= total; ++i) {
    step_++;
    d->Fix((float)i / (float)total);
    const bool report = (i % info_every == 0) || i == total;
    d->WillReport(report && !info_mode_.empty());
    if (d->Calculate() != kNormal) {
      finish_dumps(0);
      return kErr;
    }
    if (report) info_out();
    if ((i % dump_every == 0) || i == total) dump_out();
  }
  const int rc = finish_dumps(0);
  log().flush();
  return rc;
}

int Driver::runfunc(std::string func) {
  Dynamics* d = current();
  if (!d) {
    log() << "Error: no system set, runfunc commands not available\n";
    return kErr;
  }
  d->Datas = &datas;
  d->Vars = &vars;
  if (!inited_[name_]) {
    log() << "Warning: Initialization function called before \"run\"\n";
    d->Initialize();
    inited_[name_] = true;
  }
  return d->RunFunc(func);
}

int Driver::device(std::string args) {
  int id = 0;
  args >> id;
  if (gs_set_device(id) != GS_OK) {
    log() << "Error: gpu device change operation unsuccessful!\n";
    return kErr;
  }
  log() << "gpu device changes to device " << id << "\n";
  return kNormal;
}

}  // namespace gsfe
