// The reference program with the B200 backend: the reference's own main (src/app/main.cpp) and
// run_program (src/app/run.cpp:457-611), whose BackendFactory parameter takes b200_backend_factory.
// Command line as the reference's, plus --device b200 (FP64 form) or --device b200-mixed.
#include <unistd.h>

#include <iostream>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "app/cli.hpp"
#include "app/run.hpp"
#include "b200_backend.hpp"

int main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  std::optional<spodvr::BackendFactory> backend;
  for (std::size_t i = 0; i + 1 < args.size(); ++i) {
    if (args[i] != "--device") continue;
    if (args[i + 1] == "b200" || args[i + 1] == "b200-mixed") {
      const auto precision =
          args[i + 1] == "b200" ? spodvr::b200::Precision::Fp64 : spodvr::b200::Precision::Mixed;
      backend = spodvr::b200::b200_backend_factory(precision, 0);
      args[i + 1] = "cpu";  // the set-up runs on the host as for any backend; the step runs on the B200
    }
  }
  spodvr::CommandLine command_line;
  try {
    command_line = spodvr::parse_command_line(args);
  } catch (const std::invalid_argument& e) {
    std::cerr << "spodvr_b200: " << e.what() << "\n\n" << spodvr::usage();
    return 2;
  }
  if (command_line.help) {
    std::cout << spodvr::usage() << "  --device b200 | b200-mixed  propagate on the B200 (FP64 | mixed form)\n";
    return 0;
  }
  const spodvr::ProgramInfo program{SPODVR_VERSION, "spodvr_b200"};
  const bool color = !command_line.no_color && isatty(STDOUT_FILENO) != 0;
  return spodvr::run_program(command_line, std::cout, std::cerr, color, program, backend);
}
