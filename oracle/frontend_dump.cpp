// Test driver (CPU only): runs the first pass of the reference's own generated parser
// (bison.cu + lex.yy.c, linked from the reference build's objects) over a script and
// prints the statements that libalenka_b200.so's emit_* boundary captured from its
// grammar actions, in alk_parse_dump's format. tests/test_frontend.py compares that with
// the engine parser's rendering of the same script. Nothing runs on a device.
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

struct yy_buffer_state;
yy_buffer_state* yy_scan_string(const char* s);
void yy_delete_buffer(yy_buffer_state* b);
int yyparse();
extern bool scan_state;
extern "C" int alk_frontend_dump(char* out, int out_len);
extern "C" void alk_frontend_reset(void);

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: frontend_dump <script file>\n");
    return 2;
  }
  std::ifstream f(argv[1]);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string script = ss.str();
  alk_frontend_reset();
  scan_state = 0;  // the first pass: grammar actions only record
  yy_buffer_state* b = yy_scan_string(script.c_str());
  const int rc = yyparse();
  yy_delete_buffer(b);
  if (rc) {
    std::printf("PARSE ERROR\n");
    return 1;
  }
  const int n = alk_frontend_dump(nullptr, 0);
  std::vector<char> out((size_t)n + 1);
  alk_frontend_dump(out.data(), n + 1);
  std::fwrite(out.data(), 1, (size_t)n, stdout);
  alk_frontend_reset();
  return 0;
}
