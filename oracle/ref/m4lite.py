"""A small m4 macro processor: enough of GNU m4 to expand the reference's
Fortran templates (define, ifelse, include, dnl, `quotes', $1..$9, $#, $0,
$*, $@, # comments), which the reference's build expands with
`m4 -DFORTDIR=... -DPDAT_FORTDIR=...` (cmake/SetupM4.cmake).  This image
has no m4.

    python m4lite.py -DNAME=value ... file.m4 > file.f

TEST INFRASTRUCTURE ONLY: part of the recipe that builds the reference into
oracle/_ref/.
"""
import sys

LQ, RQ = "`", "'"


def _is_name_start(c):
    return c.isalpha() or c == "_"


def _is_name_char(c):
    return c.isalnum() or c == "_"


class M4:
    def __init__(self, defines=None):
        self.macros = dict(defines or {})
        self.builtins = {"define", "ifelse", "include", "dnl", "undefine"}
        self.s = ""
        self.i = 0

    # -- input stack: pushing text back means splicing it before the cursor
    def push(self, text):
        self.s = text + self.s[self.i:]
        self.i = 0

    def _quoted(self):
        """Consume a quoted string at the cursor; return its text with the
        outer quotes removed."""
        assert self.s[self.i] == LQ
        depth, j = 1, self.i + 1
        out = []
        while depth:
            if j >= len(self.s):
                raise ValueError("unterminated quote")
            c = self.s[j]
            if c == LQ:
                depth += 1
            elif c == RQ:
                depth -= 1
                if depth == 0:
                    break
            out.append(c)
            j += 1
        self.i = j + 1
        return "".join(out)

    def _name(self):
        j = self.i
        while j < len(self.s) and _is_name_char(self.s[j]):
            j += 1
        n = self.s[self.i:j]
        self.i = j
        return n

    def _collect_args(self):
        """Arguments of a macro call, the cursor just past '(': leading
        whitespace skipped, one level of quotes removed, macros in the
        arguments expanded."""
        args, cur, depth = [], [], 0
        skipping = True
        while True:
            if self.i >= len(self.s):
                raise ValueError("unterminated argument list")
            c = self.s[self.i]
            if skipping and c in " \t\n":
                self.i += 1
                continue
            skipping = False
            if c == LQ:
                cur.append(self._quoted())
            elif c == "#":
                j = self.s.find("\n", self.i)
                j = len(self.s) if j < 0 else j + 1
                cur.append(self.s[self.i:j])
                self.i = j
            elif _is_name_start(c):
                n = self._name()
                if self._expandable(n):
                    self._call(n)
                else:
                    cur.append(n)
            elif c == "(":
                depth += 1
                cur.append(c)
                self.i += 1
            elif c == ")":
                if depth == 0:
                    self.i += 1
                    args.append("".join(cur))
                    return args
                depth -= 1
                cur.append(c)
                self.i += 1
            elif c == "," and depth == 0:
                args.append("".join(cur))
                cur = []
                skipping = True
                self.i += 1
            else:
                cur.append(c)
                self.i += 1

    def _expandable(self, n):
        if n in self.macros:
            return True
        if n in self.builtins:
            # define/ifelse/include/undefine are recognised only with
            # arguments; dnl always
            return n == "dnl" or self.s[self.i:self.i + 1] == "("
        return False

    def _call(self, n):
        """Expand macro n (cursor after its name) and push the result back."""
        if n == "dnl":
            j = self.s.find("\n", self.i)
            self.i = len(self.s) if j < 0 else j + 1
            return
        args = []
        if self.s[self.i:self.i + 1] == "(":
            self.i += 1
            args = self._collect_args()
        if n == "define":
            self.macros[args[0]] = args[1] if len(args) > 1 else ""
            return
        if n == "undefine":
            self.macros.pop(args[0], None)
            return
        if n == "include":
            with open(args[0]) as fh:
                self.push(fh.read())
            return
        if n == "ifelse":
            while len(args) >= 3:
                if args[0] == args[1]:
                    self.push(args[2])
                    return
                if len(args) <= 4:
                    if len(args) == 4:
                        self.push(args[3])
                    return
                args = args[3:]
            return
        self.push(self._substitute(self.macros[n], n, args))

    @staticmethod
    def _substitute(body, name, args):
        out, k = [], 0
        while k < len(body):
            c = body[k]
            if c == "$" and k + 1 < len(body):
                d = body[k + 1]
                if d.isdigit():
                    idx = int(d)
                    out.append(name if idx == 0 else (args[idx - 1] if idx <= len(args) else ""))
                    k += 2
                    continue
                if d == "#":
                    out.append(str(len(args)))
                    k += 2
                    continue
                if d == "*":
                    out.append(",".join(args))
                    k += 2
                    continue
                if d == "@":
                    out.append(",".join(LQ + a + RQ for a in args))
                    k += 2
                    continue
            out.append(c)
            k += 1
        return "".join(out)

    def expand(self, text):
        self.s, self.i = text, 0
        out = []
        while self.i < len(self.s):
            c = self.s[self.i]
            if c == LQ:
                out.append(self._quoted())
            elif c == "#":
                j = self.s.find("\n", self.i)
                j = len(self.s) if j < 0 else j + 1
                out.append(self.s[self.i:j])
                self.i = j
            elif _is_name_start(c):
                n = self._name()
                if self._expandable(n):
                    self._call(n)
                else:
                    out.append(n)
            else:
                # copy a run of ordinary characters at once
                j = self.i + 1
                while j < len(self.s) and not (_is_name_start(self.s[j]) or
                                                self.s[j] in (LQ, "#")):
                    j += 1
                out.append(self.s[self.i:j])
                self.i = j
        return "".join(out)


def expand_file(path, defines):
    with open(path) as fh:
        return M4(defines).expand(fh.read())


def main(argv):
    defines, files = {}, []
    for a in argv:
        if a.startswith("-D"):
            k, _, v = a[2:].partition("=")
            defines[k] = v
        else:
            files.append(a)
    for f in files:
        sys.stdout.write(expand_file(f, defines))


if __name__ == "__main__":
    main(sys.argv[1:])
