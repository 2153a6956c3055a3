// permutation_matrix.hpp -- the result type of the semi-local LCS path.
//
// Same public interface as the reference's PermutationMatrix
// (src/permutation_matrix.hpp:5-204): a square partial permutation kept as
// row->col and col->row arrays with -1 for "no point", built from strands by
// FromStrands (88-115), compared with == (164-173) and hashed with the
// reference's polynomial hash (192-203).  The interface is kept so that code
// written against the reference compiles unchanged; the storage and the move
// semantics are this library's own (a moved-from matrix is empty).
#pragma once

#include <cstdint>
#include <utility>

#include "slcs.h"

using int64 = signed long long;

class PermutationMatrix
{
public:
    // Empty matrix; also the error value of a failed procedure.
    PermutationMatrix() = default;

    // Owning matrix of the given size with every entry unset.
    explicit PermutationMatrix(int size) : size_(size)
    {
        if (size > 0) {
            row_to_col_ = new int[size];
            col_to_row_ = new int[size];
            owns_ = true;
            unset_all();
        }
    }

    PermutationMatrix(PermutationMatrix &&o) noexcept { take(o); }
    PermutationMatrix &operator=(PermutationMatrix &&o) noexcept
    {
        if (this != &o) {
            release();
            take(o);
        }
        return *this;
    }
    PermutationMatrix(const PermutationMatrix &) = delete;
    PermutationMatrix &operator=(const PermutationMatrix &) = delete;
    ~PermutationMatrix() { release(); }

    // Non-owning view over caller memory.
    static PermutationMatrix Preallocated(int size, int *row_to_col, int *col_to_row)
    {
        PermutationMatrix p;
        p.size_ = size;
        p.row_to_col_ = row_to_col;
        p.col_to_row_ = col_to_row;
        return p;
    }

    PermutationMatrix SameSizeEmpty() const { return PermutationMatrix(size_); }

    // The strand leaving row l on the right is column n+l; the strand leaving
    // column j at the bottom is column j; the strand id is the row.
    void init_from_strands(const int *h_strands, int m, const int *v_strands, int n)
    {
        for (int l = 0; l < m; ++l)
            if (h_strands[l] >= 0 && h_strands[l] < size_) set_point(h_strands[l], n + l);
        for (int j = 0; j < n; ++j)
            if (v_strands[j] >= 0 && v_strands[j] < size_) set_point(v_strands[j], j);
    }

    static PermutationMatrix FromStrands(const int *h_strands, int m, const int *v_strands, int n)
    {
        PermutationMatrix p(m + n);
        p.init_from_strands(h_strands, m, v_strands, n);
        return p;
    }

    int row_count() const { return size_; }
    int col_count() const { return size_; }
    int get_col(int row) const { return row_to_col_[row]; }
    int get_row(int col) const { return col_to_row_[col]; }
    const int *row_to_col() const { return row_to_col_; }
    const int *col_to_row() const { return col_to_row_; }
    bool empty() const { return size_ == 0; }

    void set_point(int row, int col)
    {
        row_to_col_[row] = col;
        col_to_row_[col] = row;
    }

    void unset_all()
    {
        for (int i = 0; i < size_; ++i) row_to_col_[i] = col_to_row_[i] = -1;
    }

    bool operator==(const PermutationMatrix &o) const
    {
        if (size_ != o.size_) return false;
        for (int i = 0; i < size_; ++i)
            if (row_to_col_[i] != o.row_to_col_[i] || col_to_row_[i] != o.col_to_row_[i]) return false;
        return true;
    }

    double similarity(const PermutationMatrix &o) const
    {
        if (size_ != o.size_ || size_ == 0) return 0.0;
        int good = 0;
        for (int i = 0; i < size_; ++i)
            good += (row_to_col_[i] == o.row_to_col_[i]) + (col_to_row_[i] == o.col_to_row_[i]);
        return double(good) / double(2 * size_);
    }

    int64 hash() const { return size_ ? slcs_permutation_hash(col_to_row_, size_) : 0; }

private:
    void take(PermutationMatrix &o)
    {
        row_to_col_ = std::exchange(o.row_to_col_, nullptr);
        col_to_row_ = std::exchange(o.col_to_row_, nullptr);
        size_ = std::exchange(o.size_, 0);
        owns_ = std::exchange(o.owns_, false);
    }
    void release()
    {
        if (owns_) {
            delete[] row_to_col_;
            delete[] col_to_row_;
        }
        row_to_col_ = col_to_row_ = nullptr;
        size_ = 0;
        owns_ = false;
    }

    int *row_to_col_ = nullptr;
    int *col_to_row_ = nullptr;
    int size_ = 0;
    bool owns_ = false;
};
