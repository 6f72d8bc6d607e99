// stand-in: the reference's inner pfor loops run serially in the oracle
#pragma once
#define pfor(counter, from, to, grain) for (int counter = from; counter < to; counter++) {
#define endpfor }
