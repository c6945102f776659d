// metropolis -- the klft `metropolis` binary (binaries/metropolis.cpp:35-92) on
// libklft_b200: `metropolis -f input.yaml`, output files as the reference's.
#include <getopt.h>

#include <cstdio>
#include <string>

#include "klft/klft.hpp"

#define HLINE "====================================================================\n"

static int parse_args(int argc, char **argv, std::string &input_file) {
  input_file = "input.yaml";
  const std::string help_string =
      "  -f <file_name> --filename <file_name>\n"
      "     Name of the input file.\n"
      "     Default: input.yaml\n"
      "  -h, --help\n"
      "     Prints this message.\n";
  static struct option long_options[] = {
      {"filename", required_argument, NULL, 'f'}, {"help", no_argument, NULL, 'h'}, {NULL, 0, NULL, 0}};
  int c, option_index = 0;
  while ((c = getopt_long(argc, argv, "f:h", long_options, &option_index)) != -1) switch (c) {
      case 'f': input_file = optarg; break;
      case 'h': printf("%s", help_string.c_str()); return -2;
      case 0: break;
      default: printf("%s", help_string.c_str()); return -1;
    }
  return 0;
}

int main(int argc, char *argv[]) {
  printf(HLINE);
  printf("Metropolis for SU(N) gauge fields\n");
  printf(HLINE);
  std::string input_file;
  int rc = parse_args(argc, argv, input_file);
  if (rc == 0) rc = klft::Metropolis(input_file);
  else if (rc == -2) rc = 0;
  return rc;
}
