// simulator.hpp - host-side session over librodgpu with the surface of the
// reference's Python simulator (src/python/rod_dynamics_py.cpp:52-91).
#pragma once
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "../../include/rodgpu.h"

namespace rgjson { struct Value; }

namespace rgsim {

class Simulator {
 public:
  Simulator(const std::string& scene_path, const std::string& init_csv_path = std::string(), bool quiet = true);
  ~Simulator();
  Simulator(const Simulator&) = delete;
  Simulator& operator=(const Simulator&) = delete;

  void step(int steps = 1);
  // Per-frame writers of the reference App (enabled by its CLI there):
  // the profile CSV (App::enableCsv / logCsvFrame, src/app/main.cpp:162-172,
  // :3276-3355) and the NSC contact network (logNetworkFrame, :3620-3700,
  // every `stride` frames, at most max_frames frames when > 0).  While either
  // is on, step(n) advances one frame per library call so every frame is
  // logged.
  void enable_csv(const std::string& path);
  void enable_network(const std::string& path, int stride = 1, int max_frames = 0);
  int rod_count() const { return n_; }
  long long frame_index() const { return frame_; }
  double dt() const { return cfg_.dt; }
  double last_ke() const { return last_ke_; }
  long long last_hit_count() const { return last_hits_; }
  const rg_step_stats& last_stats() const { return stats_; }
  const rg_config& config() const { return cfg_; }
  rg_system* handle() const { return sys_; }

  // per-rod state (read back from the device on first access after a step)
  const std::vector<double>& x() const;
  const std::vector<double>& q() const;
  const std::vector<double>& v() const;
  const std::vector<double>& w() const;
  const std::vector<double>& f() const;
  const std::vector<double>& tau() const;
  double mass(int i) const { return mass_[i]; }
  double radius(int i) const { return radius_[i]; }
  double half_height(int i) const { return half_[i]; }
  double restitution(int i) const { return rest_[i]; }
  void endpoints(int i, double a[3], double b[3]) const;

 private:
  void check(int rc, const char* what) const;
  void add_body(const rgjson::Value* b, std::vector<double>& dens);
  void push(const double x[3], const double q[4], const double v[3], const double w[3], double r, double h,
            double rho, double e, bool is_static, std::vector<double>& dens);
  void populate(const rgjson::Value& pop, std::vector<double>& dens);
  void load_csv(const std::string& path, const rgjson::Value& pop, const rgjson::Value* tmpl,
                std::vector<double>& dens);
  void random_init(const rgjson::Value& ri);
  double kinetic_energy() const;
  void sync() const;
  void log_frame();
  void com(double c[3]) const;
  double gyration_sq() const;
  double relative_motion_sq();

  bool quiet_ = true;
  rg_config cfg_{};
  rg_system* sys_ = nullptr;
  int n_ = 0;
  long long frame_ = 0;
  double last_ke_ = 0;
  long long last_hits_ = 0;
  rg_step_stats stats_{};
  bool fresh_ = true;
  std::vector<double> x_, q_, v_, w_, f_, tau_;
  std::vector<double> radius_, half_, rest_, mass_, inertia_;
  std::vector<int> static_;
  // writers
  std::unique_ptr<std::ofstream> csv_;
  bool csv_header_ = false;
  std::unique_ptr<std::ofstream> net_;
  bool net_header_ = false;
  int net_stride_ = 1, net_max_ = 0, net_written_ = 0;
  std::vector<double> last_pos_;
  double last_com_[3] = {0, 0, 0};
  bool has_last_pos_ = false;
};

}  // namespace rgsim
