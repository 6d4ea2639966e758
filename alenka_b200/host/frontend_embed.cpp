// The embedding API of alenka.h (alenka.h:30-35) with the C++ linkage the reference gives
// it: alenka.h declares these without extern "C" and the reference compiles its callers
// (main.cu, bison.cu) as C++, so a caller built from the reference's sources binds the
// mangled names defined here. They run the same code as the C entry points of
// include/alenka_b200.h (this file does not see those declarations: one name cannot have
// both linkages in one translation unit).
namespace alk {
void embed_init(char** av);
int embed_execute(char* s);
void embed_close();
int embed_file(int ac, char** av);
}  // namespace alk

void alenkaInit(char** av) { alk::embed_init(av); }
int alenkaExecute(char* s) { return alk::embed_execute(s); }
void alenkaClose() { alk::embed_close(); }
int execute_file(int ac, char** av) { return alk::embed_file(ac, av); }
