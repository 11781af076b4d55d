"""The hand-built three-rank CommPatterns of the reference's communication test
(test/mpitest_n3_communication.jl:13-73), with 0-based indices and (start, stop) slices:
per rank the data length, the pattern fields and the data every rank holds after the
exchange when each starts with data[i] = i + 1 + 100 rank."""

CASES = {
    0: dict(
        datalength=10,
        recvindices=[6, 7, 8, 9], recvranks=[1, 2], recvrankindices=[(0, 1), (1, 4)],
        sendindices=[0, 2, 0, 2, 4], sendranks=[1, 2], sendrankindices=[(0, 2), (2, 5)],
        datacomm=[1, 2, 3, 4, 5, 6, 102, 201, 202, 203],
    ),
    1: dict(
        datalength=16,
        recvindices=[10, 11, 12, 13, 14, 15], recvranks=[0, 2], recvrankindices=[(0, 2), (2, 6)],
        sendindices=[1, 1, 3, 5, 7, 9], sendranks=[0, 2], sendrankindices=[(0, 1), (1, 6)],
        datacomm=[101, 102, 103, 104, 105, 106, 107, 108, 109, 110, 1, 3, 202, 203, 204, 205],
    ),
    2: dict(
        datalength=20,
        recvindices=[7, 8, 9, 13, 14, 15, 16, 17], recvranks=[0, 1], recvrankindices=[(0, 3), (3, 8)],
        sendindices=[0, 1, 2, 1, 2, 3, 4], sendranks=[0, 1], sendrankindices=[(0, 3), (3, 7)],
        datacomm=[201, 202, 203, 204, 205, 206, 207, 1, 3, 5, 211, 212, 213, 102, 104, 106, 108, 110, 219, 220],
    ),
}


def pattern(distributed, rank):
    c = CASES[rank]
    return distributed.CommPattern(c["recvindices"], c["recvranks"], c["recvrankindices"], c["sendindices"],
                                   c["sendranks"], c["sendrankindices"])
