// solver_cavity on the B200 step: the reference CLI's arguments, steady-stop
// loop and `key: value` report (tools/lid_driven_cavity_main.cpp).
//
//   solver_cavity [config.cfg] [--steps N] [--restart path]
//                 [--checkpoint-out path] [--vtk-out path]
//                 [--device N] [--precision fp64|mixed]
//
// --device and --precision are additions.  Checkpoints are SLVCHKP1 files
// stamped with this library's build hash.
#include "orchard_b200_cases.h"

#include <iostream>
#include <stdexcept>
#include <string>

namespace {

void check(of_status s) {
  if(s != OF_OK) throw std::runtime_error(of_last_error());
}

struct Context {
  of_ctx* ctx = nullptr;
  ~Context() {
    if(ctx) of_destroy(ctx);
  }
};

const char* line_name(int line) { return line == OF_U_VERTICAL ? "u_vertical" : "v_horizontal"; }

}  // namespace

int main(int argc, char** argv) {
  try {
    std::string config_path = "benchmarks/lid_driven_cavity_re100_128.cfg";
    std::string restart_path, checkpoint_out, vtk_out;
    bool partial_run = false;
    int steps_override = 0;
    int device = 0;
    int precision = OF_FP64;
    bool config_consumed = false;
    for(int index = 1; index < argc; ++index) {
      const std::string arg = argv[index];
      const auto value = [&]() -> std::string {
        if(index + 1 >= argc) throw std::runtime_error("missing value for " + arg);
        return argv[++index];
      };
      if(arg == "--steps") {
        steps_override = std::stoi(value());
        partial_run = true;
      } else if(arg == "--restart") restart_path = value();
      else if(arg == "--checkpoint-out") checkpoint_out = value();
      else if(arg == "--vtk-out") vtk_out = value();
      else if(arg == "--device") device = std::stoi(value());
      else if(arg == "--precision") {
        const std::string p = value();
        if(p == "fp64") precision = OF_FP64;
        else if(p == "mixed") precision = OF_MIXED;
        else throw std::runtime_error("invalid precision value: " + p);
      } else if(!config_consumed && !arg.empty() && arg.rfind("--", 0) != 0) {
        config_path = arg;
        config_consumed = true;
      } else {
        throw std::runtime_error("unsupported argument: " + arg);
      }
    }

    of_cavity_config config{};
    check(of_cavity_config_load(config_path.c_str(), &config));
    Context c;
    check(of_cavity_create(&config, device, &c.ctx));
    check(of_set_precision(c.ctx, precision));
    if(!restart_path.empty()) check(of_cavity_checkpoint_load(c.ctx, restart_path.c_str(), &config, 0, nullptr));
    if(partial_run) check(of_cavity_run_steps(c.ctx, &config, steps_override, nullptr));
    else check(of_cavity_run_to_steady(c.ctx, &config, nullptr));
    if(!checkpoint_out.empty()) check(of_cavity_checkpoint_write(c.ctx, checkpoint_out.c_str(), &config, 0));
    if(!vtk_out.empty()) check(of_write_vtk(c.ctx, vtk_out.c_str()));

    of_cavity_result result{};
    check(of_cavity_finalize(c.ctx, &config, &result));
    char text[1024];
    check(of_cavity_config_describe(&config, text, sizeof(text), nullptr));
    const of_step_metrics& s = result.final_step;
    std::cout << "config_path: " << config_path << '\n';
    std::cout << "config: " << text << '\n';
    std::cout << "steps: " << s.step << '\n';
    std::cout << "time: " << s.time << '\n';
    std::cout << "dt: " << s.dt << '\n';
    std::cout << "max_cfl: " << s.max_cfl << '\n';
    std::cout << "max_velocity_change: " << s.max_velocity_change << '\n';
    std::cout << "divergence_l2: " << s.divergence_l2 << '\n';
    std::cout << "pressure_iterations: " << s.pressure_iterations << '\n';
    std::cout << "pressure_relative_residual: " << s.pressure_relative_residual << '\n';
    std::cout << "u_vertical_max: " << result.u_vertical_max << '\n';
    std::cout << "u_vertical_min: " << result.u_vertical_min << '\n';
    std::cout << "v_horizontal_max: " << result.v_horizontal_max << '\n';
    std::cout << "v_horizontal_min: " << result.v_horizontal_min << '\n';
    std::cout << "reference_dataset: " << result.reference_dataset << '\n';
    std::cout << "max_reference_relative_error: " << result.max_relative_error << '\n';
    for(const of_cavity_point& p : result.points) {
      if(p.label[0] == '\0') continue;
      std::cout << "reference_point[" << p.label << "]: line=" << line_name(p.line)
                << ", coordinate=" << p.coordinate << ", reference=" << p.reference_value
                << ", reference_lower=" << p.reference_lower_bound
                << ", reference_upper=" << p.reference_upper_bound << ", sample=" << p.sample_value
                << ", relative_error=" << p.relative_error << '\n';
    }
    if(!restart_path.empty()) std::cout << "restart_path: " << restart_path << '\n';
    if(!checkpoint_out.empty()) std::cout << "checkpoint_out: " << checkpoint_out << '\n';
    if(!vtk_out.empty()) std::cout << "vtk_out: " << vtk_out << '\n';

    if(partial_run || !config.validate_reference) {
      std::cout << "benchmark_status: skipped" << '\n';
      return 0;
    }
    if(result.reference_dataset[0] == '\0') {
      std::cout << "benchmark_status: unavailable" << '\n';
      return 1;
    }
    std::cout << "benchmark_status: " << (result.pass ? "pass" : "fail") << '\n';
    return result.pass ? 0 : 1;
  } catch(const std::exception& e) {
    std::cerr << "solver_cavity failed: " << e.what() << '\n';
    return 1;
  }
}
