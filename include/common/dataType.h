/*
 * Matrix structs of the reference's ABI (include/common/dataType.h:24-77 in
 * SingkiWong/DCU).  Field order and types are kept identical so that code
 * written against the reference passes the same structs to this library:
 * pointers first (index, data, ptr), then the int sizes.
 */
#ifndef MATRIX_DATATYPE_H
#define MATRIX_DATATYPE_H

typedef struct {
  int *mIndex;    /* column indices, nonzeroes entries            */
  double *mData;  /* values, nonzeroes entries                    */
  int *mPtr;      /* row pointers, nRow + 1 entries               */
  int nRow;
  int nCol;
  int n;          /* order of a square matrix                     */
  int nonzeroes;
} CSR_Matrix;

typedef struct {
  int *mIndex;    /* row indices, nonzeroes entries               */
  double *mData;  /* values, nonzeroes entries                    */
  int *mPtr;      /* column pointers, nCol + 1 entries            */
  int nRow;
  int nCol;
  int n;
  int nonzeroes;
} CSC_Matrix;

typedef struct {
  int nRow;
  int nCol;
  int nDIG;
  int nonzeroes;
  int *mOffset;
  double *mData;
} DIA_Matrix;

typedef struct {
  int nRow;
  int nCol;
  int nonzeroes;
  int *mIndex;
  double *mData;
} ELL_Matrix;

typedef struct {
  int n;
  int nonzeroes;
  int *mI;
  int *mJ;
  double *mV;
} COO_Matrix;

typedef struct {
  double *vect;
  int n;
} Vector;

typedef struct {
  int n;
  double *dgl;
} DIAGS;

#endif
