// BLOSUM62 in NCBIstdaa order (28 letters: -ABCDEFGHIKLMNPQRSTVWXYZU*OJ).
//
// The 22x22 block over ARNDCQEGHILKMFPSTWYVBZ is BLOSUM62 (Henikoff &
// Henikoff, PNAS 89:10915, 1992) as NCBI distributes it: it differs from the
// 1992 file only in ambiguity entries (B-Z 0, W-Z -2, Q-Z 4).  Around it the NCBIstdaa
// conventions the reference scores with (its table: gpu_blastp.c:46-75):
// the gap letter '-' (code 0) scores -128 against everything, so no word
// containing it can reach the neighbour threshold and a walk that meets it
// stops; X, U and O score -1 against every letter; '*' scores -4 against
// every letter and +1 against itself; J (I or L) has its own row.
#include <stdint.h>
#include <string.h>

namespace {

const char kNcbiStdaa[] = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ";
const char kBlockOrder[] = "ARNDCQEGHILKMFPSTWYVBZ";

const int8_t kBlock[22][22] = {
    // A   R   N   D   C   Q   E   G   H   I   L   K   M   F   P   S   T   W   Y   V   B   Z
    {  4, -1, -2, -2,  0, -1, -1,  0, -2, -1, -1, -1, -1, -2, -1,  1,  0, -3, -2,  0, -2, -1},  // A
    { -1,  5,  0, -2, -3,  1,  0, -2,  0, -3, -2,  2, -1, -3, -2, -1, -1, -3, -2, -3, -1,  0},  // R
    { -2,  0,  6,  1, -3,  0,  0,  0,  1, -3, -3,  0, -2, -3, -2,  1,  0, -4, -2, -3,  4,  0},  // N
    { -2, -2,  1,  6, -3,  0,  2, -1, -1, -3, -4, -1, -3, -3, -1,  0, -1, -4, -3, -3,  4,  1},  // D
    {  0, -3, -3, -3,  9, -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1, -3, -3},  // C
    { -1,  1,  0,  0, -3,  5,  2, -2,  0, -3, -2,  1,  0, -3, -1,  0, -1, -2, -1, -2,  0,  4},  // Q
    { -1,  0,  0,  2, -4,  2,  5, -2,  0, -3, -3,  1, -2, -3, -1,  0, -1, -3, -2, -2,  1,  4},  // E
    {  0, -2,  0, -1, -3, -2, -2,  6, -2, -4, -4, -2, -3, -3, -2,  0, -2, -2, -3, -3, -1, -2},  // G
    { -2,  0,  1, -1, -3,  0,  0, -2,  8, -3, -3, -1, -2, -1, -2, -1, -2, -2,  2, -3,  0,  0},  // H
    { -1, -3, -3, -3, -1, -3, -3, -4, -3,  4,  2, -3,  1,  0, -3, -2, -1, -3, -1,  3, -3, -3},  // I
    { -1, -2, -3, -4, -1, -2, -3, -4, -3,  2,  4, -2,  2,  0, -3, -2, -1, -2, -1,  1, -4, -3},  // L
    { -1,  2,  0, -1, -3,  1,  1, -2, -1, -3, -2,  5, -1, -3, -1,  0, -1, -3, -2, -2,  0,  1},  // K
    { -1, -1, -2, -3, -1,  0, -2, -3, -2,  1,  2, -1,  5,  0, -2, -1, -1, -1, -1,  1, -3, -1},  // M
    { -2, -3, -3, -3, -2, -3, -3, -3, -1,  0,  0, -3,  0,  6, -4, -2, -2,  1,  3, -1, -3, -3},  // F
    { -1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4,  7, -1, -1, -4, -3, -2, -2, -1},  // P
    {  1, -1,  1,  0, -1,  0,  0,  0, -1, -2, -2,  0, -1, -2, -1,  4,  1, -3, -2, -2,  0,  0},  // S
    {  0, -1,  0, -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1,  1,  5, -2, -2,  0, -1, -1},  // T
    { -3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1,  1, -4, -3, -2, 11,  2, -3, -4, -2},  // W
    { -2, -2, -2, -3, -2, -1, -2, -3,  2, -1, -1, -2, -1,  3, -3, -2, -2,  2,  7, -1, -3, -2},  // Y
    {  0, -3, -3, -3, -1, -2, -2, -3, -3,  3,  1, -2,  1, -1, -2, -2,  0, -3, -1,  4, -3, -2},  // V
    { -2, -1,  4,  4, -3,  0,  1, -1,  0, -3, -4,  0, -3, -3, -2,  0, -1, -4, -3, -3,  4,  0},  // B
    { -1,  0,  0,  1, -3,  4,  4, -2,  0, -3, -3,  1, -1, -3, -1,  0, -1, -2, -2, -2,  0,  4},  // Z
};

// J against each NCBIstdaa letter, in code order.
const int8_t kJRow[28] = {-128, -1, -3, -1, -3, -3, 0, -4, -3, 3, -3, 3, 2, -3,
                          -3, -2, -2, -2, -1, 2, -2, -1, -1, -3, -1, -4, -1, 3};

int code_of(char c) { return (int)(strchr(kNcbiStdaa, c) - kNcbiStdaa); }

}  // namespace

// Robinson & Robinson (1991) background, per 1000, in NCBIstdaa code order
// (0 for non-standard letters).
static const float kBackground[28] = {0,     78.05, 0,     19.25, 53.64, 62.95, 38.56, 73.77, 21.99, 51.42,
                                      57.44, 90.19, 22.43, 44.87, 52.03, 42.64, 51.29, 71.20, 58.41, 64.41,
                                      13.30, 0,     32.16, 0,     0,     0,     0,     0};

float bp_expected_hits_per_residue(const uint32_t* cells) {
    double h = 0.0;
    for (int a = 1; a < 28; ++a) {
        if (kBackground[a] == 0.f) continue;
        for (int b = 1; b < 28; ++b) {
            if (kBackground[b] == 0.f) continue;
            const double pab = (double)kBackground[a] * kBackground[b] * 1e-6;
            for (int c = 1; c < 28; ++c) {
                if (kBackground[c] == 0.f) continue;
                const int cell = (a - 1) * 729 + (b - 1) * 27 + (c - 1);
                h += pab * kBackground[c] * 1e-3 * (double)(cells[cell + 1] - cells[cell]);
            }
        }
    }
    return (float)h;
}

void bp_fill_matrix28(int8_t out[28 * 28]) {
    const int star = code_of('*');
    for (int a = 0; a < 28; ++a)
        for (int b = 0; b < 28; ++b) {
            int8_t v = -1;
            if (a == star || b == star) v = (a == b) ? 1 : -4;
            if (a == 0 || b == 0) v = -128;
            out[a * 28 + b] = v;
        }
    for (int i = 0; i < 22; ++i)
        for (int j = 0; j < 22; ++j)
            out[code_of(kBlockOrder[i]) * 28 + code_of(kBlockOrder[j])] = kBlock[i][j];
    const int J = code_of('J');
    for (int b = 0; b < 28; ++b) {
        out[J * 28 + b] = kJRow[b];
        out[b * 28 + J] = kJRow[b];
    }
}
