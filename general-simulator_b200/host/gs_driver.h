// gs_driver.h -- the run driver and the plugin interface of the front end.
//
// Dynamics is the reference's plugin interface (src/dynamics.h:9-25): grid,
// the shared field and variable stores, and Initialize / Calculate / RunFunc
// / Fix / Get.  Two optional hooks are added because the physics state lives
// on the device behind the C ABI: SyncToHost copies a field into the store
// before `dump` / `write` / `writehere`, and WillReport tells the plugin that
// an info line follows the next Calculate (so force means can be taken from
// the state the step starts from, as the reference reports them).  A third,
// DumpAsync, lets `dump` overlap the steps after it: the plugin snapshots the
// field on the device and returns a job that waits for the copy and fills a
// host Field, which a writer thread then writes (`set asyncdump 0` dumps
// synchronously, as the reference does).
//
// Driver is GS (src/gs.cu, src/gs.h): `sys` registry, `set`, `link`,
// `read`, `readhere`, `write`, `writehere`, `info`, `dump`, `run`, `runfunc`.
#pragma once
#include <deque>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <string>
#include <utility>

#include "gs_data.h"
#include "gs_script.h"

namespace gsfe {

class Dynamics {
 public:
  virtual ~Dynamics() = default;
  int nx = 1, ny = 1, nz = 1;
  float dx = 1, dy = 1, dz = 1;
  Store<Field>* Datas = nullptr;
  Store<std::string>* Vars = nullptr;
  virtual int Initialize() = 0;
  virtual int Calculate() = 0;
  virtual int RunFunc(std::string func) = 0;
  virtual int Fix(float progress) = 0;
  virtual std::string Get(std::string key) = 0;
  virtual int SyncToHost(const std::string& field) { (void)field; return kNormal; }
  virtual void WillReport(bool) {}
  // Start copying `field` off the device for a dump; the returned job (run on
  // another thread) waits for the copy, fills its Field and returns 0, or a
  // message.  An empty job: no asynchronous copy for this field.
  using DumpJob = std::function<std::string(Field&)>;
  virtual DumpJob DumpAsync(const std::string& field) { (void)field; return {}; }
};

// factory of the registered plugins: mart, precipitate, stress, cores, pow
std::unique_ptr<Dynamics> make_dynamics(const std::string& name);

class Driver {
 public:
  Driver();
  Store<Field> datas;
  Store<std::string> vars;
  Expressions expr;

  int set_sys(std::string args);
  int set(std::string args);
  int link(std::string args);
  int read(std::string args);
  int readhere(const std::string& name, std::string arrays);
  int write(std::string args);
  int writehere(std::string args);
  int set_info(std::string args);
  int set_dump(std::string args);
  int run(std::string args);
  int runfunc(std::string func);
  int device(std::string args);

 private:
  Dynamics* current();
  void info_out();
  void dump_out();
  void dump_field(const std::string& name, const std::string& file);
  // asynchronous dumps in flight: field name, writer (copy wait + file write)
  struct PendingDump {
    std::string name;
    std::future<std::pair<std::string, Field>> done;
  };
  std::deque<PendingDump> pending_;
  int finish_dumps(size_t keep);  // join all but `keep` of them, oldest first
  std::map<std::string, std::unique_ptr<Dynamics>> systems_;
  std::map<std::string, bool> inited_;
  std::string name_;
  bool binary_ = false;
  long step_ = 0;
  int info_steps_ = 0;
  std::string info_mode_;
  std::string dump_folder_;
  int dump_steps_ = 0;
  std::string dump_mode_;
};

}  // namespace gsfe
