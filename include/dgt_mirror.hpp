// C++ mirror of the reference's hot-path classes on top of the dgt C ABI, for callers that
// used them directly.  Same class names, constructor arguments and method names as the
// reference; the MPI communicator argument is replaced by the virtual grid size, because
// the whole grid lives on one device.  Errors are reported the reference's way only in
// spirit: instead of exit()/MPI_Abort() every method throws dgt::Error carrying the status.
//
//   pblasDecomposer            include/pblasDecomposition.hpp:21-37
//   BlockSequentialDecomposer  include/2DBlockSequentialDecomposition.hpp:12-36
//   Summa25Decomposer          include/25DCannon.hpp:30-92
//
// All buffers are device pointers.  Local buffers are owned by the caller (the reference's
// decomposers own theirs; here the caller decides where the virtual ranks' tiles live).
#ifndef DGT_MIRROR_HPP
#define DGT_MIRROR_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "dgt.h"

namespace dgt {

struct Error : std::runtime_error {
    dgt_status status;
    Error(dgt_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

inline void check(dgt_handle_t h, dgt_status s) {
    if (s != DGT_SUCCESS)
        throw Error(s, std::string(dgt_status_string(s)) + ": " + (h ? dgt_last_error(h) : ""));
}

// Owning handle (cublasCreate/cublasDestroy replacement, src/25DCannon.cpp:66, :381).
class Context {
  public:
    Context() { check(nullptr, dgt_create(&h_)); }
    ~Context() { dgt_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    dgt_handle_t get() const { return h_; }

  private:
    dgt_handle_t h_ = nullptr;
};

// copyBlock<T> for the reference's two instantiations, double and float
// (src/Transfers/sharedTransfers.cpp:29-63, :87-88): one strided copy on the handle's
// stream.  Unlike the reference, a null pointer is an error rather than a printed no-op.
inline void copyBlock(dgt_handle_t h, long long rows, long long columns, const double* src, double* dst,
                      long long ldSource, long long ldDestination, bool columnMajor = true) {
    check(h, dgt_copy_block(h, rows, columns, src, dst, ldSource, ldDestination, columnMajor));
}
inline void copyBlock(dgt_handle_t h, long long rows, long long columns, const float* src, float* dst,
                      long long ldSource, long long ldDestination, bool columnMajor = true) {
    check(h, dgt_copy_block_f32(h, rows, columns, src, dst, ldSource, ldDestination, columnMajor));
}

// ScaLAPACK block-cyclic layout of an M x N matrix on a dRow x dCol grid (row-major ranks).
class pblasDecomposer {
  public:
    int M, N, Mb, Nb, dRow, dCol, size;
    std::vector<int> localRows, localColumns, myBlocks;  // per virtual rank

    pblasDecomposer(dgt_handle_t h, int M_, int N_, int Mb_, int Nb_, int dRow_, int dCol_)
        : M(M_), N(N_), Mb(Mb_), Nb(Nb_), dRow(dRow_), dCol(dCol_), size(dRow_ * dCol_), h_(h) {
        if (M <= 0 || N <= 0 || Mb <= 0 || Nb <= 0 || dRow <= 0 || dCol <= 0)
            throw Error(DGT_ERROR_INVALID_VALUE, "pblasDecomposer: bad sizes or grid");
        const int gridRows = (M + Mb - 1) / Mb, gridCols = (N + Nb - 1) / Nb;
        for (int r = 0; r < size; ++r) {
            int pr = r / dCol, pc = r % dCol;
            localRows.push_back(dgt_numroc(M, Mb, pr, 0, dRow));
            localColumns.push_back(dgt_numroc(N, Nb, pc, 0, dCol));
            int b = 0;
            for (int i = pr; i < gridRows; i += dRow) b += (gridCols - pc + dCol - 1) / dCol;
            myBlocks.push_back(b);
        }
    }
    std::vector<int64_t> lld() const {
        std::vector<int64_t> v;
        for (int r : localRows) v.push_back(r > 0 ? r : 1);
        return v;
    }
    // scatterMatrix(sender, global, local) for every rank at once (pblasDecomposition.cpp:73-148)
    void scatterMatrix(const double* globalMatrix, double* const* localMatrices) const {
        auto l = lld();
        check(h_, dgt_pack_block_cyclic(h_, M, N, Mb, Nb, dRow, dCol, globalMatrix, M, localMatrices, l.data()));
    }
    // gatherMatrix(receiver, global, local) (pblasDecomposition.cpp:150-221)
    void gatherMatrix(double* globalMatrix, const double* const* localMatrices) const {
        auto l = lld();
        check(h_, dgt_unpack_block_cyclic(h_, M, N, Mb, Nb, dRow, dCol, globalMatrix, M, localMatrices, l.data()));
    }

  private:
    dgt_handle_t h_;
};

// 2D block layout: A row panels (full K), B column panels, C blocks; remainder rows and
// columns go to the last grid row / column.
class BlockSequentialDecomposer {
  public:
    int M, N, K, numberOfDevices, dRow = 1, dCol = 1;
    bool colMajor;
    std::vector<int> localM, localN;

    BlockSequentialDecomposer(dgt_handle_t h, int M_, int N_, int K_, int P, bool colMajor_ = true)
        : M(M_), N(N_), K(K_), numberOfDevices(P), colMajor(colMajor_), h_(h) {
        check(h_, dgt_block2d_grid(P, &dRow, &dCol));
        for (int r = 0; r < P; ++r) {
            int i = r / dCol, j = r % dCol;
            localM.push_back(M / dRow + (i + 1 == dRow ? M % dRow : 0));
            localN.push_back(N / dCol + (j + 1 == dCol ? N % dCol : 0));
        }
    }
    void deliverMatrix(const double* A, const double* B, const double* C, double* const* lA, double* const* lB,
                       double* const* lC) const {
        check(h_, dgt_pack_block2d(h_, M, N, K, numberOfDevices, colMajor, A, B, C, lA, lB, lC));
    }
    void gatherResult(double* C, const double* const* lC) const {
        check(h_, dgt_unpack_block2d(h_, M, N, numberOfDevices, colMajor, C, lC));
    }

  private:
    dgt_handle_t h_;
};

// 2.5D Cannon on a virtual dRow x dCol x c grid (dRow == dCol, M == N == K, as the
// reference's constructor enforces: src/25DCannon.cpp:7-23).  The stack-0 tiles
// (localA/B/C of ranks 0..p*p-1) are the caller's device buffers of (M/p)^2 doubles.
class Summa25Decomposer {
  public:
    long long M, N, K, localM, localN, localK;
    int dRow, dCol, c, pc, pc3;

    Summa25Decomposer(dgt_handle_t h, long long M_, long long N_, long long K_, int dRow_, int dCol_, int c_)
        : M(M_), N(N_), K(K_), dRow(dRow_), dCol(dCol_), c(c_), h_(h) {
        if (M != N || M != K) throw Error(DGT_ERROR_INVALID_VALUE, "2.5D Cannon supports only M = N = K");
        if (dRow != dCol) throw Error(DGT_ERROR_INVALID_VALUE, "2.5D Cannon supports only dRow = dCol");
        if (c <= 0 || dRow % c != 0) throw Error(DGT_ERROR_INVALID_VALUE, "stack depth must divide the grid side");
        if (M % dRow != 0) throw Error(DGT_ERROR_INVALID_VALUE, "M must be a multiple of the grid side");
        pc = dRow;
        pc3 = dRow / c;
        localM = M / dRow;
        localN = N / dCol;
        localK = K / dRow;
    }
    // decompose2D(0, A, B, C, aTile, bTile, cTile) for every stack-0 rank (src/25DCannon.cpp:87-149)
    void decompose2D(const double* A, const double* B, const double* C, double* const* aTiles,
                     double* const* bTiles, double* const* cTiles) const {
        check(h_, dgt_pack_cannon2d(h_, M, dRow, A, B, C, aTiles, bTiles, cTiles));
    }
    // multiply(TransA, TransB, ..., alpha, beta): skew, rotations and stack reduction as
    // one in-device schedule (src/25DCannon.cpp:286-375)
    void multiply(char TransA, char TransB, const double* const* aTiles, const double* const* bTiles,
                  double* const* cTiles, double alpha, double beta, dgt_fp64_mode mode = DGT_FP64_NATIVE,
                  int slices = 7) const {
        check(h_, dgt_cannon25d(h_, M, dRow, c, TransA, TransB, alpha, aTiles, bTiles, beta, cTiles, mode, slices));
    }
    // reorderMatrix(0, C, cTile) (src/25DCannon.cpp:231-284)
    void reorderMatrix(double* C, const double* const* cTiles) const {
        check(h_, dgt_unpack_cannon2d(h_, M, dRow, C, cTiles));
    }

  private:
    dgt_handle_t h_;
};

}  // namespace dgt

#endif
