// solver_taylor_green on the B200 step: the reference CLI's arguments and its
// `key: value` report (tools/taylor_green_main.cpp), so that harness scripts
// written against the reference parse this output unchanged.
//
//   solver_taylor_green [config.cfg] [--vtk-out path] [--backend cpu]
//                       [--device N] [--precision fp64|mixed]
//                       [--checkpoint-out path] [--restart path]
//
// --device, --precision, --checkpoint-out and --restart are additions; the
// Taylor-Green checkpoint uses the SLVCHKP1 framing with a TGCF config section.
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

}  // namespace

int main(int argc, char** argv) {
  try {
    std::string config_path = "benchmarks/taylor_green_128.cfg";
    std::string vtk_out, backend_override, checkpoint_out, restart_path;
    int device = 0;
    int precision = OF_FP64;
    bool config_consumed = false;
    for(int index = 1; index < argc; ++index) {
      const std::string arg = argv[index];
      const auto value = [&]() -> std::string {
        if(index + 1 >= argc) throw std::runtime_error("missing value for " + arg);
        return argv[++index];
      };
      if(arg == "--vtk-out") vtk_out = value();
      else if(arg == "--backend") backend_override = value();
      else if(arg == "--device") device = std::stoi(value());
      else if(arg == "--checkpoint-out") checkpoint_out = value();
      else if(arg == "--restart") restart_path = value();
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

    of_tg_config config{};
    check(of_tg_config_load(config_path.c_str(), &config));
    if(!backend_override.empty()) {
      if(backend_override == "cpu") config.backend = OF_BACKEND_CPU;
      else if(backend_override == "metal") config.backend = OF_BACKEND_METAL;
      else throw std::runtime_error("invalid Taylor-Green backend value: " + backend_override);
    }
    Context c;
    check(of_tg_create(&config, device, &c.ctx));
    check(of_set_precision(c.ctx, precision));
    of_tg_result result{};
    if(restart_path.empty()) {
      check(of_tg_run(c.ctx, &config, &result));
    } else {
      // continue a checkpointed run up to final_time
      check(of_tg_checkpoint_load(c.ctx, restart_path.c_str(), &config, 0, nullptr));
      int total = 0;
      check(of_tg_case(&config, nullptr, nullptr, nullptr, &total));
      of_step_metrics m{};
      check(of_state_download(c.ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &m));
      if(total > m.step) check(of_tg_run_steps(c.ctx, &config, total - m.step, nullptr));
      check(of_tg_finalize(c.ctx, &config, &result));
    }
    if(!checkpoint_out.empty()) check(of_tg_checkpoint_write(c.ctx, checkpoint_out.c_str(), &config, 0));
    if(!vtk_out.empty()) check(of_write_vtk(c.ctx, vtk_out.c_str()));

    char text[1024];
    check(of_tg_config_describe(&config, text, sizeof(text), nullptr));
    const of_step_metrics& s = result.final_step;
    std::cout << "config_path: " << config_path << '\n';
    std::cout << "config: " << text << '\n';
    std::cout << "backend_used: cpu" << '\n';
    std::cout << "accelerator_name: " << result.accelerator_name << '\n';
    if(result.elapsed_seconds > 0.0) std::cout << "backend_elapsed_seconds: " << result.elapsed_seconds << '\n';
    std::cout << "steps: " << s.step << '\n';
    std::cout << "time: " << s.time << '\n';
    std::cout << "dt: " << s.dt << '\n';
    std::cout << "max_cfl: " << s.max_cfl << '\n';
    std::cout << "max_velocity_change: " << s.max_velocity_change << '\n';
    std::cout << "divergence_l2: " << s.divergence_l2 << '\n';
    std::cout << "max_divergence_l2: " << s.max_divergence_l2 << '\n';
    std::cout << "pressure_iterations: " << s.pressure_iterations << '\n';
    std::cout << "pressure_relative_residual: " << s.pressure_relative_residual << '\n';
    std::cout << "initial_kinetic_energy: " << result.initial_kinetic_energy << '\n';
    std::cout << "final_kinetic_energy: " << result.final_kinetic_energy << '\n';
    std::cout << "reference_dataset: " << result.reference_dataset << '\n';
    std::cout << "exact_kinetic_energy: " << result.exact_kinetic_energy << '\n';
    std::cout << "normalized_energy_error: " << result.normalized_energy_error << '\n';
    std::cout << "velocity_relative_l2_error: " << result.velocity_relative_l2_error << '\n';
    if(!restart_path.empty()) std::cout << "restart_path: " << restart_path << '\n';
    if(!checkpoint_out.empty()) std::cout << "checkpoint_out: " << checkpoint_out << '\n';
    if(!vtk_out.empty()) std::cout << "vtk_out: " << vtk_out << '\n';

    if(!config.validate_energy) {
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
    std::cerr << "solver_taylor_green failed: " << e.what() << '\n';
    return 1;
  }
}
