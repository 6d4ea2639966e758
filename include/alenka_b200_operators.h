/* Operator-level boundary of libalenka_b200.so: the reference's own C++ entry points,
 * exported with the reference's signatures and global state so that its generated script
 * front end (bison.cu / lex.yy.c from bison.y and fl.l, its main.cu CLI and its
 * alenka.h embedding callers) links against this library unchanged and runs on the
 * B200 engine. Unlike include/alenka_b200.h this is a C++ interface (the reference's is),
 * declared here as the reference declares it; every symbol is defined in
 * alenka_b200/host/frontend_abi.cpp, frontend_embed.cpp and csrc/frontend_state.cu.
 *
 * Execution model, as the reference's drivers run it (bison.y:295-515): the first parse
 * pass (scan_state == 0) calls the statement emitters, which capture the queued
 * arguments as one statement each; load_vars() then runs the captured script on the
 * engine of the embedding session (the current directory's catalog); the second pass's
 * emitters (scan_state == 1) only clear the queues. Errors reach error_cb as
 * process_error sends them (operators.cu:2751-2765). */
#ifndef ALENKA_B200_OPERATORS_H
#define ALENKA_B200_OPERATORS_H
#ifdef __cplusplus
#include <cstddef>
#include <ctime>
#include <map>
#include <queue>
#include <string>

typedef long long int int_type; /* cm.h:56 */
typedef double float_type;      /* cm.h:57 */
struct col_data {               /* cm.h:661-664 */
  unsigned int col_type;
  unsigned int col_length;
};
class CudaSet; /* cm.h:681: only named by varNames; this engine keeps its own variables */

/* Argument queues the grammar actions fill (cm.h:66-78, operators.cu:24-41). */
extern std::queue<std::string> op_type, op_value, op_sort, op_presort, col_aliases;
extern std::queue<int_type> op_nums;
extern std::queue<float_type> op_nums_f;
extern std::queue<unsigned int> op_nums_precision;
extern std::queue<std::string> op_join;
extern std::queue<char> join_type, join_eq_type;
extern unsigned int sel_count, join_cnt, distinct_cnt, join_col_cnt, join_tab_cnt, tab_cnt;
extern std::map<unsigned int, unsigned int> join_and_cnt;
extern bool op_case;

/* State the drivers read or reset (cm.cu:44-79, operators.cu:42-47, merge.cu:29). */
extern std::map<std::string, CudaSet*> varNames;
extern std::map<std::string, std::map<std::string, col_data> > data_dict;
extern size_t process_count, alloced_sz, total_buffer_size;
extern bool verbose, interactive, ssd, delta, star, save_dict;
extern unsigned int prs, hash_seed;
extern std::clock_t tot_disk;

/* Expression and argument emitters (operators.h:14-42, operators.cu:62-360). */
void emit(const char* s, ...);
void emit_mul();
void emit_add();
void emit_minus();
void emit_distinct();
void emit_cast();
void emit_year();
void emit_month();
void emit_day();
void emit_div();
void emit_and();
void emit_eq();
void emit_neq();
void emit_or();
void emit_cmp(const int val);
void emit_var(const char* s, const int c, const char* f, const char* ref, const char* ref_name);
void emit_var_asc(const char* s);
void emit_var_desc(const char* s);
void emit_name(const char* name);
void emit_count();
void emit_sum();
void emit_average();
void emit_min();
void emit_max();
void emit_string(const char* str);
void emit_number(const int_type val);
void emit_float(const float_type val);
void emit_decimal(const char* str);
void emit_sel_name(const char* name);
void emit_limit(const int val);
void emit_varchar(const char* s, const int c, const char* f, const int d, const char* ref, const char* ref_name,
                  const char* encoding);
void emit_vardecimal(const char* s, const int c, const char* f, const int scale, const int precision);
void emit_join_tab(const char* s, const char tp);
void emit_sort(const char* s, const int p);
void emit_presort(const char* s);
void emit_case();
void emit_fieldname(const char* name1, const char* name2);
void emit_string_grp(const char* str, const char* str_grp);

/* Statement emitters (operators.h:43-71; operators.cu:797, 1641, 1801, 2306, 2410-2552). */
void emit_union(const char* s, const char* f1, const char* f2);
void emit_load(const char* s, const char* f, const int d, const char* sep);
void emit_load_binary(const char* s, const char* f, const int d);
void emit_store(const char* s, const char* f, const char* sep);
void emit_store_binary(const char* s, const char* f, const bool append);
void emit_filter(char* s, char* f);
void emit_delete(const char* f);
void emit_insert(const char* f, const char* s);
void emit_order(const char* s, const char* f, const int e, const int ll = 0);
void emit_group(const char* s, const char* f, const int e);
void emit_select(const char* s, const char* f, const int grp_cnt);
void emit_join(const char* s, const char* j1, const int grp, const int start_seg, const int end_seg);
void emit_display(const char* s, const char* sep);
void emit_show_tables();
void emit_describe_table(const char* table_name);
void emit_drop_table(const char* table_name);
void emit_create_bitmap_index(const char* index_name, const char* ltable, const char* rtable, const char* rcolumn,
                              const char* lid, const char* rid);
void emit_create_index(const char* index_name, const char* table, const char* column);
void emit_create_interval(const char* interval_name, const char* table, const char* lcolumn, const char* rcolumn);

/* Driver support (operators.h:11-13, 60, 70; cm.cu:3184, 4057-4114). */
void clean_queues();
void load_vars();
void yyerror(char* s, ...);
void process_error(const int severity, const std::string err);
size_t getFreeMem();
void load_col_data(std::map<std::string, std::map<std::string, col_data> >& data_dict, std::string file_name);
void save_col_data(std::map<std::string, std::map<std::string, col_data> >& data_dict, std::string file_name);

/* alenka.h:30-35 with its C++ linkage (the C entry points are in alenka_b200.h). */
void alenkaInit(char** av);
int alenkaExecute(char* s);
void alenkaClose();
int execute_file(int ac, char** av);

#endif /* __cplusplus */

#ifdef __cplusplus
extern "C" {
#endif
/* Front-end test support: render the statements the first pass captured (the format of
 * alk_parse_dump; returns the length), and drop them. No counterpart in the reference. */
int alk_frontend_dump(char* out, int out_len);
void alk_frontend_reset(void);
#ifdef __cplusplus
}
#endif
#endif /* ALENKA_B200_OPERATORS_H */
