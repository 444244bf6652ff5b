/*
 * Command-line driver of the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 *   emp_oracle_cli <puzzle.csv> new_strategy [--strategy=basic|spiral]
 *                  [--results=<results.bin>] [--limit=<nodes>]
 *   emp_oracle_cli <puzzle.csv> glutton_max [--budget=<placements>]
 *
 * It prints the same lines as the reference's features (include/emp_strategy.h:
 * 360-414, include/CUDA_glutton_max.h:181-212) so the golden test files can be
 * checked line by line.  Puzzle files use the reference CSV format
 * (include/emp_pieces_parser.h:53-101).
 */
#include "emp_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int parse(const char *path, uint32_t *w, uint32_t *h, uint8_t *col)
{
    FILE *f = fopen(path, "r");
    if (!f) { fprintf(stderr, "Unable to open file \"%s\" for reading\n", path); return -1; }
    char line[512];
    if (!fgets(line, sizeof(line), f) || strncmp(line, "Width,Height", 12)) { fclose(f); return -2; }
    if (!fgets(line, sizeof(line), f) || sscanf(line, "%u,%u", w, h) != 2) { fclose(f); return -3; }
    if (!fgets(line, sizeof(line), f) || strncmp(line, "I,N,E,S,O", 9)) { fclose(f); return -4; }
    uint32_t cnt = 0;
    while (fgets(line, sizeof(line), f)) {
        unsigned id, n, e, s, o;
        if (sscanf(line, "%u,%u,%u,%u,%u", &id, &n, &e, &s, &o) == 5) {
            if (id < 1 || id > 256) { fclose(f); return -5; }
            col[4 * (id - 1) + 0] = (uint8_t)n;
            col[4 * (id - 1) + 1] = (uint8_t)e;
            col[4 * (id - 1) + 2] = (uint8_t)s;
            col[4 * (id - 1) + 3] = (uint8_t)o;
            ++cnt;
        }
    }
    fclose(f);
    return cnt == *w * *h ? 0 : -6;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <puzzle.csv> new_strategy|glutton_max [options]\n", argv[0]);
        return 2;
    }
    uint32_t w = 0, h = 0;
    static uint8_t col[4 * 256];
    if (parse(argv[1], &w, &h, col)) { fprintf(stderr, "bad puzzle file\n"); return 1; }
    char err[256];
    op_puzzle *p = op_puzzle_create(w, h, col, err, sizeof(err));
    if (!p) { fprintf(stderr, "%s\n", err); return 1; }
    const char *strategy = "basic", *results = NULL;
    unsigned long long limit = 0, budget = 0;
    for (int i = 3; i < argc; ++i) {
        if (!strncmp(argv[i], "--strategy=", 11)) strategy = argv[i] + 11;
        else if (!strncmp(argv[i], "--results=", 10)) results = argv[i] + 10;
        else if (!strncmp(argv[i], "--limit=", 8)) limit = strtoull(argv[i] + 8, NULL, 10);
        else if (!strncmp(argv[i], "--budget=", 9)) budget = strtoull(argv[i] + 9, NULL, 10);
    }
    if (!strcmp(argv[2], "new_strategy")) {
        uint32_t order[256];
        if (!strcmp(strategy, "spiral")) op_order_spiral(w, h, order);
        else op_order_basic(w, h, order);
        size_t cap = 1 << 22;
        char *log = (char *)malloc(cap);
        op_bt_result r;
        op_bt_run(p, order, limit, &r, results, log, cap);
        fputs(log, stdout);
        printf("End of algorithm\n");
        printf("Total situations explored : %llu\n", (unsigned long long)r.nodes);
        printf("Nb solutions : %llu\n", (unsigned long long)r.solutions);
        free(log);
    } else if (!strcmp(argv[2], "glutton_max")) {
        op_gm_result r;
        op_gm_run(p, budget, 0, &r);
        printf("Launch kernels\n");
        if (r.status == 2) {
            printf("Empty stack\n");
        } else {
            int width = snprintf(NULL, 0, "%u", w * h) + 1;
            char *board = (char *)malloc((size_t)width * w * h + 1);
            memset(board, '-', (size_t)width * w * h);
            board[width * w * h] = 0;
            uint32_t upto = r.status == 0 ? r.level : r.level + 1;
            for (uint32_t l = 0; l < upto && l < w * h; ++l) {
                uint32_t pi = r.played[l];
                if (pi == 0xFFFFFFFFu) continue;
                uint32_t pos = pi & 0xFF, piece = (pi >> 8) & 0xFF, o = pi >> 16;
                char cell[16];
                snprintf(cell, sizeof(cell), "%*u%c", width - 1, piece + 1, "NESW"[o & 3]);
                memcpy(board + (size_t)pos * width, cell, (size_t)width);
            }
            printf("Situation with stack played info:\n%s\n", board);
            free(board);
        }
        printf("Max level : %u\nPlacements : %llu\n", r.max_level, (unsigned long long)r.placements);
    } else {
        fprintf(stderr, "unknown feature %s\n", argv[2]);
        op_puzzle_destroy(p);
        return 2;
    }
    op_puzzle_destroy(p);
    return 0;
}
